"""The reference's output files, written by mahyco_b200.output after a run
on the GPU, against the reference's own files.

For every sequential golden dataset the final Ensight state
(output/depouillement: ensight.case, the geometry and each post-processed
variable) must have the digest of the reference's file once round-off noise
is removed (tests/ensight_digest.py), and the EnvSummation curves
(output/courbes/gnuplot) must match the reference's to the bounds of
test_gpu_golden.py.
"""
import glob
import json
import os
import sys

import numpy as np
import pytest

from mahyco_b200.case import params_from_dict

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import ensight_digest  # noqa: E402

GOLDEN = sorted(p for p in glob.glob(os.path.join(HERE, "golden", "CAS_*.json"))
                if json.load(open(p)).get("ensight_sha256") and "restart_at" not in json.load(open(p))["extra"])


@pytest.mark.gpu
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-5] for p in GOLDEN])
def test_gpu_outputs_match_reference_files(path, tmp_path):
    from mahyco_b200.output import run_case
    g = json.load(open(path))
    r = run_case(params_from_dict(g["params"]), {"env_names": g["env_names"], "output_vars": g["output_vars"],
                                                 "save_init": g.get("save_init", False),
                                                 "init_fields": g.get("init_fields", {}),
                                                 "mesh_file": g.get("mesh_file")}, str(tmp_path))
    assert r["scalars"]["status"] == 8, r["scalars"]  # stopped at the final time
    dep = tmp_path / "depouillement"
    bad = [k for k, v in g["ensight_sha256"].items() if ensight_digest.digest(str(dep / k)) != v]
    assert not bad, bad
    # the curves to the golden's own bounds (test_gpu_golden.py)
    tol = g["extra"].get("tol", 1e-13)
    ttol = g["extra"].get("time_tol", 1e-14)
    for key, ref in g["time_history"].items():
        ours = np.loadtxt(tmp_path / "courbes" / "gnuplot" / key, ndmin=2)
        ref = np.array(ref)
        assert ours.shape == ref.shape, (key, ours.shape, ref.shape)
        np.testing.assert_allclose(ours[:, 0], ref[:, 0], rtol=ttol, atol=0)
        var = next(v for v in ("CellMass", "Pressure", "Density", "InternalEnergy") if key.startswith(v + "_"))
        np.testing.assert_allclose(ours[:, 1], ref[:, 1], rtol=g["extra"].get("tol_var", {}).get(var, tol), atol=0)
