"""The CPU oracle against the reference's own non-regression time histories
and, for the sequential datasets, its final Ensight files.

tests/golden/<case>.json holds the parameters parsed from the case's
Donnees.arc and the EnvSummation curves the reference wrote
(NONREGRESSION/<case>/output/courbes/gnuplot), made by make_golden.py.
Sequential runs agree to ~1e-14 (the residue is the summation order of the
per-environment averages); the multi-rank reference runs (CAS_Sedov on 8
ranks, the third-order cases on 4) sum their averages per rank and their
node sums in per-rank order, hence the looser bounds.
"""
import glob
import json
import os
import sys

import numpy as np
import pytest

from mahyco_b200.case import params_from_dict
from mahyco_b200.output import write_ensight

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import ensight_digest  # noqa: E402
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "CAS_*.json")))
VARS = ("CellMass", "Pressure", "Density", "InternalEnergy")


def run_oracle(g, cr_pow=False, out_dir=None):
    """The golden's case on the oracle; with ``out_dir``, also its Ensight
    files (initial step with save-init, final step) written there."""
    from tests.oracle import Oracle
    p = params_from_dict(g["params"])
    o = Oracle(p, cr_pow=cr_pow)
    for name, values in g.get("init_fields", {}).items():
        o.set_initial_field(name, values)
    if "restart_at" in g["extra"]:
        o.set_option("restart_at", g["extra"]["restart_at"])
    assert o.init() == 0
    mf = g.get("mesh_file")
    if out_dir and g.get("save_init"):
        write_ensight(o, out_dir, g["output_vars"], 0.0, mesh_file=mf)
    nlines = max(len(v) for v in g["time_history"].values())
    period = p.time_history_period if p.time_history_period > 0 else 10
    assert o.run(max_iter=2 * period * nlines) == 0
    if out_dir:
        t = o.scalar("time")
        if g.get("save_init"):
            write_ensight(o, out_dir, g["output_vars"], t, 1, [0.0, t], mesh_file=mf)
        else:
            write_ensight(o, out_dir, g["output_vars"], t, mesh_file=mf)
    return p, o.time_history()


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-5] for p in GOLDEN])
@pytest.mark.parametrize("cr_pow", [False, True], ids=["glibc_pow", "cr_pow"])
def test_oracle_matches_reference_goldens(path, cr_pow, tmp_path):
    g = json.load(open(path))
    if cr_pow and g["params"].get("sans_lagrange"):
        # an advection without Lagrange phase calls no power that reaches
        # the state (the characteristic length is never read)
        pytest.skip("no power on the path")
    multi = g["extra"].get("mpi_ranks", 1) > 1
    tol = g["extra"].get("tol", 5e-12 if multi else 1e-13)
    ttol = 1e-13 if multi else 1e-14  # the time: a sum of deltat, per-rank orders move it by ulps
    ttol = g["extra"].get("time_tol", ttol)
    tol_var = g["extra"].get("tol_var", {})
    exact = g["extra"].get("exact_lines_cr_pow" if cr_pow else "exact_lines", 0)
    # the correctly rounded run (the only run of an advection, which calls
    # no power) also writes the final state in the reference's Ensight
    # format, compared with the digests of the reference's own files
    # (sequential datasets; tests/ensight_digest.py)
    outputs = ((cr_pow or g["params"].get("sans_lagrange")) and bool(g.get("ensight_sha256"))
               and "restart_at" not in g["extra"])
    p, th = run_oracle(g, cr_pow, str(tmp_path) if outputs else None)
    if outputs:
        dep = tmp_path / "depouillement"
        bad = [k for k, v in g["ensight_sha256"].items() if ensight_digest.digest(str(dep / k)) != v]
        assert not bad, bad
    for e, env in enumerate(g["env_names"]):
        for q, var in enumerate(VARS):
            key = f"{var}_{env}"
            if key not in g["time_history"]:
                continue
            ref = np.array(g["time_history"][key])
            assert len(th) >= len(ref), (key, len(th), len(ref))
            ours = th[: len(ref)]
            np.testing.assert_allclose(ours[:, 0], ref[:, 0], rtol=ttol, atol=0)
            # curves that stay 0 (the Fictif pressure and energy) must be 0
            den = np.where(ref[:, 1] == 0.0, 1.0, np.abs(ref[:, 1]))
            rel = np.abs(ours[:, 1 + 5 * e + q] - ref[:, 1]) / den
            assert rel.max() <= tol_var.get(var, tol), (key, rel.max(), int(rel.argmax()))
            # the lines the reference's own arithmetic reproduces bit for bit
            assert np.array_equal(ours[:exact, 1 + 5 * e + q], ref[:exact, 1]), key
