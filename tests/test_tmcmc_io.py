"""The reference's TMCMC files (parameter file, generation databases, run
record, posterior statistics) written around the in-process driver.  Host
logic only: no GPU."""
import math
import shutil
import subprocess

import numpy as np
import pytest

from gliomasolver_b200.tmcmc import TMCMCOptions, tmcmc
from gliomasolver_b200.tmcmc_io import (Checkpointer, curgen_db_text, load_checkpoint, parse_par, posterior_rows,
                                        runinfo_text, statistics_text, write_reference_outputs)

# A parameter file in the reference's syntax: tabs and spaces, comment lines,
# an inline comment, a commented-out key, B1 before B10, a parameter (B3)
# without its own range, and MaxChainLength written as 1e6 (read with %d).
PAR = """# settings

Nth\t\t12
MaxStages\t1000
PopSize\t\t300
#PopSize 99
MinChainLength\t1
MaxChainLength\t1e6
Bdef             -1\t    2
B0\t\t-8.5   -3.25
B1\t\t-5.75   -1.5
B2      \t 6.5    9.75
B4              -0.5   -0.25
B10\t\t-3.0   -2.25
B11\t\t-2.0   -1.0
TolCOV\t\t0.5  # keep
bbeta\t\t0.04
#seed\t\t0
seed\t\t1234
opt.MaxIter\t7
opt.Tol\t\t1e-9
opt.Display\t1
iplot\t\t0
"""


def test_parameter_file_is_read_as_the_reference_reads_it():
    par = parse_par(PAR)
    assert (par.nth, par.max_stages, par.pop_size) == (12, 1000, 300)
    assert (par.min_chain, par.max_chain) == (1, 1)
    assert (par.tol_cov, par.bbeta, par.seed) == (0.5, 0.04, 1234)
    assert (par.opt_max_iter, par.opt_tol, par.opt_display) == (7, 1e-9, 1)
    assert (par.lb, par.ub) == (-1.0, 2.0)
    np.testing.assert_array_equal(par.lower[[0, 1, 2, 4, 10, 11]], [-8.5, -5.75, 6.5, -0.5, -3.0, -2.0])
    np.testing.assert_array_equal(par.upper[[0, 1, 2, 4, 10, 11]], [-3.25, -1.5, 9.75, -0.25, -2.25, -1.0])
    # no "B3" line, and "B5".."B9" only occur in no line either: Bdef
    for i in (3, 5, 6, 7, 8, 9):
        assert (par.lower[i], par.upper[i]) == (-1.0, 2.0)
    opts = par.options()
    assert (opts.pop_size, opts.max_stages, opts.tol_cov, opts.bbeta, opts.seed) == (300, 1000, 0.5, 0.04, 1234)


def test_parameter_file_defaults():
    par = parse_par("# nothing set\n")
    assert (par.nth, par.max_stages, par.pop_size, par.min_chain, par.max_chain) == (4, 20, 1024, 0, 1000000)
    assert (par.tol_cov, par.bbeta, par.seed) == (1.0, 0.2, 280675)
    np.testing.assert_array_equal(par.lower, [-6.0] * 4)
    np.testing.assert_array_equal(par.upper, [6.0] * 4)


def _gauss(th):
    return -0.5 * np.sum(((th - 0.2) / 0.15) ** 2, axis=1)


@pytest.fixture(scope="module")
def run():
    return tmcmc(_gauss, [-1.0, -1.0, -1.0], [1.0, 1.0, 1.0], TMCMCOptions(pop_size=200, seed=3))


def test_driver_records_every_generation(run):
    gens = len(run.stages)
    assert gens == len(run.p) and run.p[0] == 0.0 and run.p[-1] == 1.0 and run.p_next == 1.0
    assert len(run.uniques) == len(run.coef_var) == len(run.log_selection) == len(run.mean_theta) == gens
    assert run.uniques[0] == 200 and all(1 <= u <= 200 for u in run.uniques)
    # the last generation is weighed toward the exponent that follows it (1):
    # uniform weights, COV 0 (up to the rounding of their mean), log-evidence
    # increment 0
    assert abs(run.coef_var[-1]) < 1e-12 and run.log_selection[-1] == 0.0
    total = 0.0
    for v in run.log_selection:
        total += v
    assert total == run.log_evidence
    theta, F = run.stages[-1]
    np.testing.assert_array_equal(theta, run.theta)
    np.testing.assert_array_equal(F, run.loglik)
    np.testing.assert_allclose(run.mean_theta[-1], theta.mean(axis=0), rtol=0, atol=1e-14)
    dev = theta - theta.mean(axis=0)
    np.testing.assert_allclose(run.ss, dev.T @ dev / len(theta), rtol=1e-12, atol=1e-15)
    # the posterior of a Gaussian likelihood on a wide box: mean 0.2, sd 0.15
    assert np.all(np.abs(run.mean_theta[-1] - 0.2) < 0.05)


def test_generation_cap_counts_the_prior_generation():
    r = tmcmc(_gauss, [-1.0, -1.0], [1.0, 1.0], TMCMCOptions(pop_size=64, max_stages=2, seed=1))
    assert len(r.stages) == 2 and len(r.p) == 2 and r.p[-1] < 1.0 < 1.0 + r.p_next


def test_generation_database_layout():
    theta = np.array([[0.5, -1.25, 3.0], [1e-3, 2.0 / 3.0, -7.0]])
    F = np.array([-12.5, -0.1])
    text = curgen_db_text(theta, F)
    lines = text.splitlines()
    assert lines[0] == "%20.16f %20.16f %20.16f %20.16f" % (0.5, -1.25, 3.0, -12.5)
    assert lines[1] == "%20.16f %20.16f %20.16f %20.16f" % (1e-3, 2.0 / 3.0, -7.0, -0.1)
    assert all(len(f) >= 18 for ln in lines for f in ln.split())
    back = np.array([[float(t) for t in ln.split()] for ln in lines])
    np.testing.assert_allclose(back[:, :3], theta, rtol=0, atol=1e-16)
    np.testing.assert_allclose(back[:, 3], F, rtol=0, atol=1e-16)


def test_run_record_layout(run):
    gen = len(run.stages) - 1
    text = runinfo_text(run, 1000, 200)
    lines = text.split("\n")
    d = 3
    assert lines[0] == "Gen=" and lines[1] == str(gen)
    assert lines[2] == "CoefVar[1000]="
    # the reference's extraction reads p[Gen] at line Gen + 1005 (1-based)
    # of a 1000-generation record and tests it against 1
    assert lines[1003] == "p[1000]="
    assert lines[gen + 1005 - 1] == "1.0000000000000000"
    assert int(float(lines[gen + 1005 - 1])) == 1
    assert lines[gen + 1005] == "1.0000000000000000"             # p[Gen + 1]
    assert lines[gen + 1005 + 1] == "0.0000000000000000"
    off = 2 + 1 + 1000 + 1 + 1000
    assert lines[off] == "currentuniques[1000]="
    assert [int(v) for v in lines[off + 1:off + 1 + gen + 1]] == run.uniques
    off += 1001
    assert lines[off] == "logselection[1000]="
    off += 1001
    assert lines[off] == "acceptance[1000]="
    assert float(lines[off + 1]) == 1.0
    assert float(lines[off + 1 + gen]) == run.uniques[-1] / 200
    off += 1001
    assert lines[off] == "SS[3][3]="
    np.testing.assert_allclose(np.array(lines[off + 1:off + 10], dtype=float), run.ss.ravel(), atol=1e-16)
    off += 10
    assert lines[off] == "meantheta[1000][3]"
    assert len(lines) == off + 1 + 1000 * d + 1 and lines[-1] == ""
    np.testing.assert_allclose(np.array(lines[off + 1 + gen * d:off + 1 + gen * d + d], dtype=float),
                               run.mean_theta[-1], atol=1e-16)
    with pytest.raises(ValueError):
        runinfo_text(run, gen, 200)


def test_posterior_and_statistics_follow_the_extraction_script():
    # log parameters (Dw, rho, c = Tend^2 rho) and a log-likelihood
    rho = np.array([0.02, 0.05, 0.01, 0.03])
    tend = np.array([100.0, 60.0, 250.0, 120.0])
    Dw = np.array([0.1, 0.2, 0.05, 0.3])
    theta = np.log(np.stack([Dw, rho, tend ** 2 * rho], axis=1))
    F = np.array([-30.0, -12.0, -12.0, -40.0])
    rows = posterior_rows(theta, F)
    assert rows[0][1] == "0.02" and rows[0][2] == "100" and rows[0][3] == ("%20.16f" % -30.0).strip()
    for r, t in zip(rows, tend):
        assert abs(float(r[2]) - t) <= 1e-4 * t
    stats = statistics_text(rows).split("\n")
    assert stats[0] == "MAP  | " + " ".join(rows[1][:3])          # first of the two best
    vals = np.array([[float(t) for t in r[:3]] for r in rows])
    mean = ["%.4f" % m for m in vals.mean(axis=0)]
    assert stats[1] == "mean | " + " ".join(mean)
    std = ["%.4f" % math.sqrt(((float(m) - vals[:, j]) ** 2).sum() / 3) for j, m in enumerate(mean)]
    assert stats[2] == "std  | " + " ".join(std) + " "


@pytest.mark.skipif(shutil.which("awk") is None, reason="no awk")
def test_posterior_fields_match_awk():
    rng = np.random.default_rng(0)
    theta = rng.normal(0.0, 2.0, (50, 5))
    F = rng.normal(-20.0, 5.0, 50)
    db = curgen_db_text(theta, F)
    out = subprocess.run(["awk", "{for(k=1;k<NF;k++) $k=exp($k); $3=sqrt($3/$2); print}"], input=db,
                         capture_output=True, text=True, check=True).stdout
    assert out == "".join(" ".join(r) + "\n" for r in posterior_rows(theta, F))


def test_write_reference_outputs(tmp_path, run):
    par = parse_par("Nth 3\nMaxStages 30\nPopSize 200\n")
    write_reference_outputs(run, tmp_path / "out", par)
    gen = len(run.stages) - 1
    names = sorted(p.name for p in (tmp_path / "out").iterdir())
    assert names == sorted(["curgen_db_%03d.txt" % g for g in range(gen + 1)]
                           + ["runinfo.txt", "fitness.txt", "posterior.txt", "statistics.txt"])
    last = (tmp_path / "out" / ("curgen_db_%03d.txt" % gen)).read_text()
    assert last == curgen_db_text(*run.stages[-1])
    assert len(last.splitlines()[0].split()) - 1 == 3
    assert (tmp_path / "out" / "fitness.txt").read_text() == "%f\n" % run.log_evidence
    assert (tmp_path / "out" / "runinfo.txt").read_text() == runinfo_text(run, 30, 200)


def test_write_reference_outputs_without_a_parameter_file(tmp_path, run):
    write_reference_outputs(run, tmp_path, posterior=False)
    gen = len(run.stages) - 1
    assert (tmp_path / "runinfo.txt").read_text() == runinfo_text(run, max(gen + 1, 20), 200)
    assert not (tmp_path / "posterior.txt").exists()


class _Stop(Exception):
    pass


def test_a_resumed_run_equals_the_uninterrupted_run(tmp_path):
    lower, upper = [-1.0, -1.0, -1.0], [1.0, 1.0, 1.0]
    opts = TMCMCOptions(pop_size=150, seed=5)
    full = tmcmc(_gauss, lower, upper, opts, on_generation=Checkpointer(tmp_path / "a"))
    assert len(full.stages) > 3 and full.p[-1] == 1.0
    ck = Checkpointer(tmp_path / "b")

    def stop_after_generation_2(rec, rng_state):
        ck(rec, rng_state)
        if len(rec.stages) == 3:
            raise _Stop

    with pytest.raises(_Stop):
        tmcmc(_gauss, lower, upper, opts, on_generation=stop_after_generation_2)
    mid = load_checkpoint(tmp_path / "b")
    assert len(mid.result.stages) == 3 and len(mid.result.p) == 3
    assert "p[20]=" in (tmp_path / "b" / "runinfo.txt").read_text() and not (tmp_path / "b" / "fitness.txt").exists()
    resumed = tmcmc(_gauss, lower, upper, opts, on_generation=Checkpointer(tmp_path / "b"), start=mid)
    assert np.array_equal(resumed.theta, full.theta) and np.array_equal(resumed.loglik, full.loglik)
    assert resumed.p == full.p and resumed.p_next == full.p_next
    assert resumed.log_evidence == full.log_evidence and resumed.evaluations == full.evaluations
    assert resumed.acceptance == full.acceptance and resumed.uniques == full.uniques
    assert resumed.log_selection == full.log_selection and resumed.coef_var == full.coef_var
    assert np.array_equal(resumed.ss, full.ss)
    files = sorted(q.name for q in (tmp_path / "a").iterdir())
    assert files == sorted(q.name for q in (tmp_path / "b").iterdir())
    for name in files:
        if name != "tmcmc_state.npz":
            assert (tmp_path / "a" / name).read_bytes() == (tmp_path / "b" / name).read_bytes(), name
    # resuming a finished run evaluates nothing more and gives the same result
    again = tmcmc(_gauss, lower, upper, opts, start=load_checkpoint(tmp_path / "a"))
    assert again.evaluations == full.evaluations and np.array_equal(again.theta, full.theta)
    assert again.log_evidence == full.log_evidence and again.p == full.p
