"""The native driver (rochpl_b200/cli/hplb_main.cpp, built as rochpl_b200/hplb)
against the Python one on the CPU: `hplb --list` prints the sweep without a
GPU, and it must list the same tests (T/V code, N, NB, P, Q, run or skip) in
the same order as rochpl_b200.driver.sweep for the same HPL.dat or command
line, and reject the same inputs with the same messages."""
import os
import subprocess

import pytest

from rochpl_b200.driver import skipped, sweep, tv_code
from rochpl_b200.hpl import HplInputError, parse_cli, parse_hpl_dat

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "rochpl_b200", "hplb")


@pytest.fixture(scope="module")
def cli():
    from rochpl_b200.build import build

    build()
    if not os.path.exists(CLI):
        pytest.fail("rochpl_b200/hplb was not built")
    return CLI


def _dat(ns="1000 2000", nbs="128", pmap="1", ps="1 2", qs="1 1", thr="16.0", pf="0 2",
         nbmin="16", ndiv="2", rf="1", bc="0 3", depth="1", swap="1", l1="0", u="0", eq="0",
         dev="6"):
    def cnt(v):
        return str(len(v.split()))

    return "\n".join([
        "HPLinpack benchmark input file", "test", "HPL.out      output file name (if any)",
        f"{dev}            device out (6=stdout,7=stderr,file)",
        f"{cnt(ns)}            # of problems sizes (N)", f"{ns}     Ns",
        f"{cnt(nbs)}            # of NBs", f"{nbs}          NBs",
        f"{pmap}            PMAP process mapping (0=Row-,1=Column-major)",
        f"{cnt(ps)}            # of process grids (P x Q)", f"{ps}          Ps", f"{qs}          Qs",
        f"{thr}         threshold", f"{cnt(pf)}            # of panel fact", f"{pf}            PFACTs",
        f"{cnt(nbmin)}            # of recursive stopping criterium", f"{nbmin}           NBMINs",
        f"{cnt(ndiv)}            # of panels in recursion", f"{ndiv}            NDIVs",
        f"{cnt(rf)}            # of recursive panel fact.", f"{rf}            RFACTs",
        f"{cnt(bc)}            # of broadcast", f"{bc}          BCASTs",
        f"{cnt(depth)}            # of lookahead depth", f"{depth}            DEPTHs",
        f"{swap}            SWAP (0=bin-exch,1=long,2=mix)", "64           swapping threshold",
        f"{l1}            L1 in (0=transposed,1=no-transposed) form",
        f"{u}            U  in (0=transposed,1=no-transposed) form",
        f"{eq}            Equilibration (0=no,1=yes)", "8            memory alignment in double (> 0)",
    ]) + "\n"


def _expected(cfg):
    lines = [f"{tv_code(a, bc, cfg.pmap)} {n} {a.nb} {p} {q} {'skip' if skipped(p, q, a) else 'run'}"
             for n, p, q, bc, a in sweep(cfg)]
    return lines


def _listed(cli, args, tmp_path=None, dat=None):
    if dat is not None:
        f = tmp_path / "HPL.dat"
        f.write_text(dat)
        args = ["-i", str(f)] + args
    r = subprocess.run([cli, "--list"] + args, capture_output=True, text=True, timeout=60)
    return r


@pytest.mark.parametrize("kw", [
    {},
    {"pmap": "0", "bc": "0 1 2 3 4 9", "pf": "0 1 2 7", "rf": "2 1"},
    {"ns": "0 100 31 4096", "nbs": "1 64 4096", "nbmin": "4 200", "ndiv": "2 3", "ps": "1", "qs": "1"},
    {"thr": "-1", "dev": "7"},
])
def test_hpl_dat_sweep_matches(cli, tmp_path, kw):
    dat = _dat(**kw)
    cfg = parse_hpl_dat(dat)
    r = _listed(cli, [], tmp_path, dat)
    assert r.returncode == 0, r.stderr
    out = r.stdout.splitlines()
    assert out[:-1] == _expected(cfg)
    thr, iters = out[-1].split()[1], out[-1].split()[3]
    assert float(thr) == cfg.thrsh and int(iters) == 1


@pytest.mark.parametrize("argv", [
    ["-N", "2000", "-NB", "256"],
    ["-N", "5000", "-NB", "512", "-P", "2", "-Q", "1", "-it", "3"],
    ["-p", "1", "-q", "1", "-f", "0.5", "-N", "77"],
])
def test_command_line_sweep_matches(cli, argv):
    cfg = parse_cli(argv)
    r = _listed(cli, argv)
    assert r.returncode == 0, r.stderr
    out = r.stdout.splitlines()
    assert out[:-1] == _expected(cfg)
    assert int(out[-1].split()[3]) == max(cfg.iters, 1)


@pytest.mark.parametrize("kw", [
    {"ns": "-5"}, {"nbs": "0"}, {"ps": "0 1"}, {"qs": "1 0"}, {"nbmin": "0"}, {"ndiv": "1"},
    {"depth": "0"}, {"depth": "-1"}, {"swap": "0"}, {"u": "1"}, {"eq": "1"},
])
def test_hpl_dat_rejections_match(cli, tmp_path, kw):
    dat = _dat(**kw)
    with pytest.raises(HplInputError) as e:
        parse_hpl_dat(dat)
    r = _listed(cli, [], tmp_path, dat)
    assert r.returncode == 1
    assert r.stderr.strip() == str(e.value)


def test_truncated_hpl_dat_and_bad_flags(cli, tmp_path):
    dat = "\n".join(_dat().splitlines()[:10]) + "\n"
    with pytest.raises(HplInputError) as e:
        parse_hpl_dat(dat)
    r = _listed(cli, [], tmp_path, dat)
    assert r.returncode == 1 and r.stderr.strip() == str(e.value)
    for argv, msg in ((["-N", "0"], "Illegal value for N. Exiting ..."),
                      (["-NB", "-3"], "Illegal value for NB. Exiting ..."),
                      (["-P", "0"], "Illegal value for P. Exiting ...")):
        r = _listed(cli, argv)
        assert r.returncode == 1 and r.stderr.strip() == msg


def test_help(cli):
    r = subprocess.run([cli, "--help"], capture_output=True, text=True, timeout=30)
    assert r.returncode == 0 and r.stdout.startswith("usage: hplb")
