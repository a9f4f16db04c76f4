"""Solver-side helpers that batch the model evaluations of lcurve_re's solvers.

levmarq_solver's Jacobian (new_scripts/levmarq_solver.cpp:789-886) makes 2 x npar
light-curve calls per iteration, one after another. Here every perturbed model
of a round goes to the engine in one batched call (lcg_light_curve_batch), and
the finite-difference scheme is the reference's: central differences where both
steps stay inside the bounds, else one-sided (backward at an upper bound, half
the range when both sides would leave it), steps halved when an evaluation
fails, non-finite derivatives set to zero. The reference divides a first
backward step by sign * (p' - p) = +h (levmarq_solver.cpp:843-849), which
gives that column the derivative's opposite sign; that is kept, so a solver
driven by this Jacobian takes the reference's steps. The scheme is pinned to
the reference's own executable: evaluated through the compiled reference, it
reproduces the uncertainties and correlations lcurve_levmarq prints from the
covariance of its Jacobian, on a model that runs every branch
(tests/test_solvers.py).

Precision: on a mixed-precision engine context a round of perturbed models is
one graph-captured batch. On an FP64 context lcg_light_curve_batch evaluates
the models of the round through the bit-identical FP64 single-model path,
concurrently on up to eight worker contexts (their latency-bound pipelines
overlap on the GPU), with the same results as single calls.
"""
import numpy as np


def residuals(calc, data):
    """compute_residuals (levmarq_solver.cpp:695-704): sqrt(w) (flux - fit) / sigma,
    with sigma = 1e-10 where ferr <= 0 and w = 1 where weight <= 0."""
    sigma = np.where(data["ferr"] > 0.0, data["ferr"], 1e-10)
    w = np.where(data["weight"] > 0.0, data["weight"], 1.0)
    return np.sqrt(w) * (data["flux"] - calc) / sigma


def engine_evaluator(engine, data, scale=True, sfac=None):
    """An evaluator for jacobian(): the models' light curves over data, in one
    batched call on a resident copy of the points. Returns (calc rows, ok)."""
    engine.set_data(data)
    base = np.ones(5) if sfac is None else np.asarray(sfac, dtype=np.float64)

    def evaluate(models):
        sf = np.tile(base, (len(models), 1))
        calc, _, _, _, status = engine.light_curve_batch_resident(
            models, scale=scale, rdata=True, sfac=sf)
        calc = np.array(calc, copy=True)
        ok = (np.asarray(status) == 0) & np.all(np.isfinite(calc), axis=1)
        return calc, ok
    return evaluate


def jacobian(evaluate, model, names, data, steps=None, limits=None, central=True,
             fd_step_rel=1.2e-4, fd_step_min=1e-10, resid0=None):
    """J[i, j] = d r_i / d p_j by finite differences (compute_jacobian,
    levmarq_solver.cpp:789-886) for the parameters `names` of `model`, the
    perturbed models of each round evaluated by one call of evaluate(models)
    -> (calc rows, ok flags). steps[j] <= 0 (or None) means
    fd_step_rel |p_j| + fd_step_min; limits[j] = (lo, hi) bounds (default
    unbounded). resid0: residuals at the model (computed when needed)."""
    names = list(names)
    npar = len(names)
    pars = np.array([model[n] for n in names], dtype=np.float64)
    steps = np.zeros(npar) if steps is None else np.asarray(steps, dtype=np.float64)
    lim = [(-np.inf, np.inf)] * npar if limits is None else list(limits)
    h = np.where(steps > 0.0, steps, fd_step_rel * np.abs(pars) + fd_step_min)

    def with_par(j, v):
        m = model.copy()
        m[names[j]] = v
        return m

    def run(items):
        """items: list of (key, model); returns {key: residuals or None}."""
        if not items:
            return {}
        calc, ok = evaluate([m for _, m in items])
        return {k: (residuals(calc[i], data) if ok[i] else None)
                for i, (k, _) in enumerate(items)}

    J = np.zeros((data.shape[0], npar))
    one_sided = []
    # central differences, with up to 5 halvings while both sides stay inside
    todo = {j: h[j] for j in range(npar)
            if central and pars[j] + h[j] <= lim[j][1] and pars[j] - h[j] >= lim[j][0]}
    if not central:
        one_sided = list(range(npar))
    else:
        one_sided = [j for j in range(npar) if j not in todo]
    for _ in range(5):
        if not todo:
            break
        res = run([((j, s), with_par(j, pars[j] + s * hc))
                   for j, hc in todo.items() for s in (1, -1)])
        nxt = {}
        for j, hc in todo.items():
            rp, rm = res[(j, 1)], res[(j, -1)]
            if rp is not None and rm is not None:
                d = (rp - rm) * (1.0 / (2.0 * hc))
                J[:, j] = np.where(np.isfinite(d), d, 0.0)
                continue
            hc *= 0.5
            if pars[j] + hc > lim[j][1] or pars[j] - hc < lim[j][0]:
                one_sided.append(j)
            else:
                nxt[j] = hc
        todo = nxt
    one_sided += list(todo)  # central differences that kept failing
    if not one_sided:
        return J
    if resid0 is None:
        calc, ok = evaluate([model])
        if not ok[0]:
            raise RuntimeError("the model itself does not evaluate")
        resid0 = residuals(calc[0], data)
    # one-sided: forward, backward at the upper bound, half the range if both
    # sides leave it; a failing step is halved up to 4 times, then backward
    state = {}
    for j in one_sided:
        hj, sign = h[j], 1.0
        pj = pars[j] + hj
        if pj > lim[j][1]:
            pj, sign = pars[j] - hj, -1.0
            if pj < lim[j][0]:
                hj = 0.5 * (lim[j][1] - lim[j][0])
                if hj < 1e-15:
                    continue
                pj, sign = pars[j] + hj, 1.0
        state[j] = (hj, sign, pj, sign * (pj - pars[j]), 0)
    while state:
        res = run([(j, with_par(j, st[2])) for j, st in state.items()])
        nxt = {}
        for j, (hj, sign, pj, actual, tries) in state.items():
            r = res[j]
            if r is not None:
                d = (r - resid0) * (1.0 / actual)
                J[:, j] = np.where(np.isfinite(d), d, 0.0)
            elif tries < 4:
                hj *= 0.5
                nxt[j] = (hj, sign, pars[j] + sign * hj, sign * hj, tries + 1)
            elif tries == 4 and sign > 0:
                nxt[j] = (hj, -1.0, pars[j] - hj, -hj, 5)
        state = nxt
    return J
