"""HPL.dat and command-line parsing, mirroring src/HPL_pdinfo.cpp."""
import os

import pytest

from rochpl_b200.hpl import HplInputError, parse_cli, parse_hpl_dat

HERE = os.path.dirname(os.path.abspath(__file__))


def dat(**kw):
    v = dict(n="4096", nb="256", p="1", q="1", pf="2", nbmin="32", ndiv="2", rf="2", depth="1",
             swap="1", l1="0", u="0", eq="0", nn="1", nnb="1")
    v.update(kw)
    return f"""HPLinpack benchmark input file
B200 single-process test
HPL.out      output file name (if any)
6            device out (6=stdout,7=stderr,file)
{v['nn']}            # of problems sizes (N)
{v['n']}         Ns
{v['nnb']}            # of NBs
{v['nb']}          NBs
0            PMAP process mapping (0=Row-,1=Column-major)
1            # of process grids (P x Q)
{v['p']}            Ps
{v['q']}            Qs
16.0         threshold
1            # of panel fact
{v['pf']}            PFACTs (0=left, 1=Crout, 2=Right)
1            # of recursive stopping criterium
{v['nbmin']}           NBMINs (>= 1)
1            # of panels in recursion
{v['ndiv']}            NDIVs
1            # of recursive panel fact.
{v['rf']}            RFACTs (0=left, 1=Crout, 2=Right)
1            # of broadcast
0            BCASTs (0=1rg,1=1rM,2=2rg,3=2rM,4=Lng,5=LnM)
1            # of lookahead depth
{v['depth']}            DEPTHs (>=0)
{v['swap']}            SWAP (0=bin-exch,1=long,2=mix)
64           swapping threshold
{v['l1']}            L1 in (0=transposed,1=no-transposed) form
{v['u']}            U  in (0=transposed,1=no-transposed) form
{v['eq']}            Equilibration (0=no,1=yes)
8            memory alignment in double (> 0)
"""


def test_parse_defaults():
    c = parse_hpl_dat(dat())
    assert c.ns == [4096] and c.nbs == [256] and c.thrsh == 16.0
    assert c.pfacts == [2] and c.rfacts == [2] and c.nbmins == [32] and c.ndivs == [2]
    assert c.outfile is None  # device out 6 = stdout
    algos = list(c.algos())
    assert len(algos) == 1 and algos[0].nb == 256


def test_parse_sweep():
    c = parse_hpl_dat(dat(nn="3", n="1000 2000 3000", nnb="2", nb="128 256"))
    assert c.ns == [1000, 2000, 3000] and c.nbs == [128, 256]
    assert len(list(c.algos())) == 2


@pytest.mark.parametrize("kw,msg", [
    (dict(depth="0"), "Value of DEPTH must be 1"),
    (dict(swap="0"), "Value of SWAP must be 1"),
    (dict(u="1"), "U  in no-transposed form unsupported"),
    (dict(eq="1"), "Equilibration currently unsupported"),
    (dict(n="-1"), "Value of N less than 0"),
    (dict(nb="0"), "Value of NB less than 1"),
    (dict(nbmin="0"), "Value of NBMIN less than 1"),
    (dict(ndiv="1"), "Value of NDIV less than 2"),
    (dict(nn="21"), "Number of values of N is less than 1 or greater than 20"),
])
def test_rejections_match_reference_messages(kw, msg):
    with pytest.raises(HplInputError) as e:
        parse_hpl_dat(dat(**kw))
    assert msg in str(e.value)


def test_unknown_fact_maps_to_right():
    c = parse_hpl_dat(dat(pf="7", rf="0"))
    assert c.pfacts == [2] and c.rfacts == [0]


def test_cli():
    c = parse_cli(["-N", "8192", "-NB", "512", "-it", "3"])
    assert c.ns == [8192] and c.nbs == [512] and c.iters == 3
    assert parse_cli(["-i", "HPL.dat"]) is None
    with pytest.raises(HplInputError):
        parse_cli(["-N", "0"])


_SHARED_CHILD = r"""
import json, os, sys
import torch.distributed as dist
from rochpl_b200.driver import shared_config
dist.init_process_group("gloo", init_method="env://")
rank = dist.get_rank()
# Only process 0's input exists; the other process is given a path that does not.
argv = ["-i", os.environ["DAT"] if rank == 0 else os.environ["DAT"] + ".missing"]
cfg = shared_config(argv, rank)
out = cfg if isinstance(cfg, str) else {"ns": cfg.ns, "nbs": cfg.nbs, "iters": cfg.iters}
print("RESULT " + json.dumps(out))
dist.destroy_process_group()
"""


@pytest.mark.parametrize("kw,want", [(dict(n="1000 2000", nn="2", nb="128"), None),
                                     (dict(depth="0"), "Value of DEPTH must be 1")])
def test_process_0_reads_the_input_for_every_process(tmp_path, kw, want):
    """As HPL_pdinfo: under torch.distributed, process 0 reads HPL.dat and
    every process takes its values -- or its input error -- from there."""
    import json
    import socket
    import subprocess
    import sys

    path = tmp_path / "HPL.dat"
    path.write_text(dat(**kw))
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    root = os.path.dirname(HERE)
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), DAT=str(path),
                   PYTHONPATH=root + os.pathsep + os.environ.get("PYTHONPATH", ""))
        procs.append(subprocess.Popen([sys.executable, "-c", _SHARED_CHILD], env=env, cwd=root,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    res = []
    for p in procs:
        try:
            so, se = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        assert p.returncode == 0, se[-3000:]
        res.append(json.loads([ln for ln in so.splitlines() if ln.startswith("RESULT ")][-1][7:]))
    assert res[0] == res[1]
    if want is None:
        assert res[0] == {"ns": [1000, 2000], "nbs": [128], "iters": 1}
    else:
        assert want in res[0]
