"""The reference's TMCMC files around the in-process driver.

A calibration with the reference reads ``tmcmc_glioma.par`` (engine_tmcmc.c
read_data, :26-230), writes one ``curgen_db_NNN.txt`` per generation
(tmcmc_db.c dump_curgen_db, :145-170), ``runinfo.txt`` (engine_tmcmc.c
save_runinfo, :374-408) and ``fitness.txt`` (the log evidence,
engine_tmcmc.c:1300-1309); ``extractInferenceOutput.sh`` then turns the last
generation into ``posterior.txt`` and ``statistics.txt``.  The functions here
read and write the same files, byte for byte in their layout, from a
:class:`~gliomasolver_b200.tmcmc.TMCMCResult`, so that the reference's
post-processing runs unchanged on a calibration made with
:func:`~gliomasolver_b200.tmcmc.tmcmc`::

    par = read_par("tmcmc_glioma.par")
    result = tmcmc(GliomaModel(...), par.lower, par.upper, par.options())
    write_reference_outputs(result, "run", par)

This is host-side file handling only (no device work).
"""
from __future__ import annotations

import json
import math
import os
import re
from dataclasses import dataclass, field

import numpy as np

from .tmcmc import TMCMCCheckpoint, TMCMCOptions, TMCMCResult

_INT = re.compile(r"[+-]?\d+")
_FLOAT = re.compile(r"[+-]?(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?")


def _scan(line: str, conv: str, count: int = 1):
    """sscanf(line, "%*s %d") / "%*s %lf" / "%*s %lf %lf": skip the first
    token, then convert the leading number of each following token; stops at
    the first conversion that fails (the values before it are kept)."""
    toks = line.split()[1:]
    pat = _INT if conv == "d" else _FLOAT
    out = []
    for t in toks[:count]:
        m = pat.match(t)
        if m is None:
            break
        out.append(int(m.group()) if conv == "d" else float(m.group()))
    return out


@dataclass
class TMCMCPar:
    """The settings of a ``tmcmc_glioma.par`` file, with the reference's
    defaults (engine_tmcmc.c:30-90) where the file is silent."""
    nth: int = 4
    max_stages: int = 20
    pop_size: int = 1024
    min_chain: int = 0
    max_chain: int = 1000000
    lb: float = -6.0
    ub: float = 6.0
    tol_cov: float = 1.0
    bbeta: float = 0.2
    seed: int = 280675
    opt_max_iter: int = 100
    opt_tol: float = 1e-6
    opt_display: int = 0
    iplot: int = 0
    lower: np.ndarray = field(default=None)
    upper: np.ndarray = field(default=None)

    def options(self) -> TMCMCOptions:
        return TMCMCOptions(pop_size=self.pop_size, max_stages=self.max_stages, tol_cov=self.tol_cov,
                            bbeta=self.bbeta, min_chain=self.min_chain, max_chain=self.max_chain, seed=self.seed)


def parse_par(text: str) -> TMCMCPar:
    """Read the settings from the text of a ``tmcmc_glioma.par`` file the
    way engine_tmcmc.c:94-190 does: a line starting with '#' is skipped; the
    first key (in the reference's order) that occurs anywhere in a line
    takes the number after the line's first token; ``B<i>`` is looked up as
    a substring, first matching line wins, and a parameter without one
    takes the ``Bdef`` range."""
    par = TMCMCPar()
    lines = [ln for ln in text.splitlines() if ln and not ln.startswith("#")]
    keys = (("Nth", "nth", "d"), ("MaxStages", "max_stages", "d"), ("PopSize", "pop_size", "d"),
            ("TolCOV", "tol_cov", "f"), ("bbeta", "bbeta", "f"), ("seed", "seed", "d"),
            ("opt.MaxIter", "opt_max_iter", "d"), ("opt.Tol", "opt_tol", "f"),
            ("opt.Display", "opt_display", "d"), ("iplot", "iplot", "d"), ("Bdef", None, "f"),
            ("MinChainLength", "min_chain", "d"), ("MaxChainLength", "max_chain", "d"))
    for ln in lines:
        for key, attr, conv in keys:
            if key in ln:
                if attr is None:
                    v = _scan(ln, "f", 2)
                    if len(v) > 0:
                        par.lb = v[0]
                    if len(v) > 1:
                        par.ub = v[1]
                else:
                    v = _scan(ln, conv)
                    if v:
                        setattr(par, attr, v[0])
                break
    lower = np.full(par.nth, par.lb)
    upper = np.full(par.nth, par.ub)
    for i in range(par.nth):
        tag = f"B{i}"
        for ln in lines:
            if tag in ln:
                v = _scan(ln, "f", 2)
                if len(v) > 0:
                    lower[i] = v[0]
                if len(v) > 1:
                    upper[i] = v[1]
                break
    par.lower, par.upper = lower, upper
    return par


def read_par(path) -> TMCMCPar:
    with open(path) as f:
        return parse_par(f.read())


def _lf(x: float) -> str:
    return "%.16f" % x


def curgen_db_text(theta: np.ndarray, F: np.ndarray) -> str:
    """One generation as dump_curgen_db writes it: per sample the
    coordinates and the log-likelihood, each ``%20.16lf``, separated by
    single spaces."""
    rows = []
    for x, f in zip(np.asarray(theta, dtype=np.float64), np.asarray(F, dtype=np.float64)):
        rows.append(" ".join("%20.16f" % v for v in x) + " " + "%20.16f" % f + "\n")
    return "".join(rows)


def runinfo_text(result: TMCMCResult, max_stages: int, pop_size: int = None) -> str:
    """``runinfo.txt`` after the last generation, as save_runinfo writes it
    at the end of a run: arrays of length max_stages (zero past the run);
    p[Gen + 1], where it fits, is the exponent after the last generation (1
    once the run reached it; 0 while the run goes on, as in the record the
    reference saves during a run); CoefVar[Gen + 1] is the COV objective at
    its optimum (0);
    acceptance[g] = distinct points of generation g / population size
    (engine_tmcmc.c:834-835)."""
    gen = len(result.stages) - 1
    if gen < 0:
        raise ValueError("the result holds no generation")
    if gen + 1 > max_stages:
        raise ValueError(f"{gen + 1} generations do not fit max_stages={max_stages}")
    n = pop_size if pop_size is not None else len(result.stages[0][1])
    d = result.stages[0][0].shape[1]
    coef = np.zeros(max_stages)
    p = np.zeros(max_stages)
    un = np.zeros(max_stages, dtype=np.int64)
    logsel = np.zeros(max_stages)
    acc = np.zeros(max_stages)
    mean = np.zeros((max_stages, d))
    coef[:gen + 1] = result.coef_var
    p[:gen + 1] = result.p[:gen + 1]
    if gen + 1 < max_stages and result.p_next is not None:
        p[gen + 1] = result.p_next
    un[:gen + 1] = result.uniques
    logsel[:gen + 1] = result.log_selection
    acc[:gen + 1] = np.asarray(result.uniques, dtype=np.float64) / n
    mean[:gen + 1] = np.asarray(result.mean_theta)
    out = ["Gen=\n", f"{gen}\n", f"CoefVar[{max_stages}]=\n"]
    out += [_lf(v) + "\n" for v in coef]
    out.append(f"p[{max_stages}]=\n")
    out += [_lf(v) + "\n" for v in p]
    out.append(f"currentuniques[{max_stages}]=\n")
    out += [f"{int(v)}\n" for v in un]
    out.append(f"logselection[{max_stages}]=\n")
    out += [_lf(v) + "\n" for v in logsel]
    out.append(f"acceptance[{max_stages}]=\n")
    out += [_lf(v) + "\n" for v in acc]
    out.append(f"SS[{d}][{d}]=\n")
    out += [_lf(v) + "\n" for v in np.asarray(result.ss).ravel()]
    out.append(f"meantheta[{max_stages}][{d}]\n")
    out += [_lf(v) + "\n" for v in mean.ravel()]
    return "".join(out)


def _awk_number(v: float) -> str:
    """A computed field as awk writes it back into a record: an integral
    value as an integer, otherwise CONVFMT "%.6g"."""
    if math.isfinite(v) and v == int(v) and abs(v) < 2.0 ** 53:
        return "%d" % int(v)
    return "%.6g" % v


def posterior_rows(theta: np.ndarray, F: np.ndarray):
    """The last generation as extractInferenceOutput.sh rewrites it into
    ``posterior.txt``: every parameter exp()'d, the third replaced by
    sqrt(third / second) (Tend = sqrt(c / rho)), the log-likelihood kept as
    written in the generation file.  Returns the rows as lists of fields."""
    rows = []
    for x, f in zip(np.asarray(theta, dtype=np.float64), np.asarray(F, dtype=np.float64)):
        v = [math.exp(t) for t in x]
        if len(v) >= 3:
            v[2] = math.sqrt(v[2] / v[1])
        rows.append([_awk_number(t) for t in v] + [("%20.16f" % f).strip()])
    return rows


def statistics_text(rows) -> str:
    """``statistics.txt`` of extractInferenceOutput.sh from posterior rows:
    the MAP row (the first with the largest log-likelihood) and each
    column's mean and sample standard deviation (about the mean rounded to
    4 decimals), both printed with 4 decimals."""
    vals = np.array([[float(t) for t in r] for r in rows])
    nparam = vals.shape[1] - 1
    best = 0
    for i in range(1, len(vals)):
        if vals[i, -1] > vals[best, -1]:
            best = i
    mean, std = [], []
    for j in range(nparam):
        m = "%.4f" % (vals[:, j].sum() / len(vals))
        mean.append(m)
        ss = ((float(m) - vals[:, j]) ** 2).sum()
        std.append("%.4f" % math.sqrt(ss / (len(vals) - 1)))
    return ("MAP  | " + " ".join(rows[best][:nparam]) + "\n" + "mean | " + " ".join(mean) + "\n"
            + "std  | " + " ".join(std) + " \n")


def write_reference_outputs(result: TMCMCResult, directory, par: TMCMCPar = None, posterior: bool = True):
    """Write curgen_db_000.txt .. curgen_db_<Gen>.txt, runinfo.txt and
    fitness.txt into ``directory`` (created if missing); with ``posterior``
    and a run that reached exponent 1, also posterior.txt and
    statistics.txt as extractInferenceOutput.sh makes them.  Without ``par``
    the run record has max(generations, 20) entries and the population size
    is the first generation's."""
    if par is None:
        par = TMCMCPar(max_stages=max(len(result.stages), 20), pop_size=len(result.stages[0][1]))
    os.makedirs(directory, exist_ok=True)
    for g, (theta, F) in enumerate(result.stages):
        with open(os.path.join(directory, "curgen_db_%03d.txt" % g), "w") as f:
            f.write(curgen_db_text(theta, F))
    with open(os.path.join(directory, "runinfo.txt"), "w") as f:
        f.write(runinfo_text(result, par.max_stages, par.pop_size))
    with open(os.path.join(directory, "fitness.txt"), "w") as f:
        total = 0.0
        for v in result.log_selection:
            total += v
        f.write("%f\n" % total)
    if posterior and result.p[-1] >= 1.0:
        rows = posterior_rows(*result.stages[-1])
        with open(os.path.join(directory, "posterior.txt"), "w") as f:
            f.write("".join(" ".join(r) + "\n" for r in rows))
        with open(os.path.join(directory, "statistics.txt"), "w") as f:
            f.write(statistics_text(rows))


def _atomic_write(path, write):
    tmp = f"{path}.tmp{os.getpid()}"
    try:
        with open(tmp, "wb") as f:
            write(f)
        os.replace(tmp, path)
    finally:
        if os.path.exists(tmp):
            os.remove(tmp)


STATE_FILE = "tmcmc_state.npz"
GENERATION_FILE = "tmcmc_gen_%03d.npz"


class Checkpointer:
    """An ``on_generation`` hook for :func:`~gliomasolver_b200.tmcmc.tmcmc`
    that writes, after every generation, what the reference writes during a
    run (curgen_db_<g>.txt, runinfo.txt; engine_tmcmc.c:1176-1184), the
    generation's population in binary (tmcmc_gen_<g>.npz, written once) and
    tmcmc_state.npz: the run's statistics and the random generator's state,
    from which ``load_checkpoint`` resumes the run exactly.  Every file is
    written under a temporary name and renamed, so a crash leaves either the
    previous version or the new one.  runinfo.txt holds ``max_stages`` rows
    (``par.max_stages`` when a parameter file is given), as the reference's
    reader expects (engine_tmcmc.c:393-394).  After the last generation it
    also writes fitness.txt (and, with ``posterior``, posterior.txt and
    statistics.txt)."""

    def __init__(self, directory, par: TMCMCPar = None, posterior: bool = True, max_stages: int = None):
        self.directory = os.fspath(directory)
        self.par = par
        self.max_stages = par.max_stages if par is not None else (max_stages or TMCMCPar().max_stages)
        self.posterior = posterior
        os.makedirs(self.directory, exist_ok=True)

    def __call__(self, result: TMCMCResult, rng_state: dict):
        g = len(result.stages) - 1
        par = self.par if self.par is not None else TMCMCPar(max_stages=max(self.max_stages, g + 1),
                                                              pop_size=len(result.stages[0][1]))
        db = curgen_db_text(*result.stages[g])
        _atomic_write(os.path.join(self.directory, "curgen_db_%03d.txt" % g), lambda f: f.write(db.encode()))
        theta, F = result.stages[g]
        _atomic_write(os.path.join(self.directory, GENERATION_FILE % g),
                      lambda f: np.savez(f, theta=theta, F=F))
        text = runinfo_text(result, par.max_stages, par.pop_size)
        _atomic_write(os.path.join(self.directory, "runinfo.txt"), lambda f: f.write(text.encode()))
        arrays = {"p": np.asarray(result.p, dtype=np.float64),
                  "acceptance": np.asarray(result.acceptance, dtype=np.float64),
                  "uniques": np.asarray(result.uniques, dtype=np.int64),
                  "coef_var": np.asarray(result.coef_var, dtype=np.float64),
                  "log_selection": np.asarray(result.log_selection, dtype=np.float64),
                  "mean_theta": np.asarray(result.mean_theta, dtype=np.float64),
                  "ss": np.asarray(result.ss, dtype=np.float64),
                  "evaluations": np.int64(result.evaluations),
                  "rng_state": np.frombuffer(json.dumps(rng_state).encode(), dtype=np.uint8)}
        _atomic_write(os.path.join(self.directory, STATE_FILE), lambda f: np.savez(f, **arrays))
        if result.p_next is not None:
            write_reference_outputs(result, self.directory, par, self.posterior)


def load_checkpoint(directory) -> TMCMCCheckpoint:
    """The state a :class:`Checkpointer` left in ``directory``: pass it as
    ``tmcmc(..., start=...)`` with the same likelihood and options."""
    directory = os.fspath(directory)
    with np.load(os.path.join(directory, STATE_FILE)) as z:
        n = int(z["p"].size)
        stages = []
        for k in range(n):
            with np.load(os.path.join(directory, GENERATION_FILE % k)) as gz:
                stages.append((gz["theta"].copy(), gz["F"].copy()))
        res = TMCMCResult(stages[-1][0], stages[-1][1], [float(v) for v in z["p"]], 0.0,
                          [float(v) for v in z["acceptance"]], int(z["evaluations"]), stages=stages,
                          uniques=[int(v) for v in z["uniques"]], coef_var=[float(v) for v in z["coef_var"]],
                          log_selection=[float(v) for v in z["log_selection"]],
                          mean_theta=[row.copy() for row in z["mean_theta"]], ss=z["ss"].copy())
        rng_state = json.loads(bytes(z["rng_state"]).decode())
    return TMCMCCheckpoint(res, rng_state)
