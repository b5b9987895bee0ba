"""The .arc reader against a dataset written in the reference's format."""
import os

import pytest

from mahyco_b200.case import read_arc, params_from_dict, params_to_dict

HERE = os.path.dirname(os.path.abspath(__file__))
ARC = os.path.join(HERE, "golden", "bisod_remap_superbee.arc")


def test_read_arc_values():
    p, info = read_arc(ARC)
    assert info["env_names"] == ["LEFT", "RIGHT"]
    assert info["timeloop"] == "MahycoLoop"
    assert (p.dim, p.nx, p.ny, p.nz) == (3, 64, 8, 8)
    assert (p.lx, p.ly, p.lz) == (1.0, 0.25, 0.25)
    assert p.nb_env == 2 and p.cas_model == 1 and p.cas_test == 13
    assert p.env[0].densite_initiale == 1.0 and p.env[1].pression_initiale == 0.1
    assert p.env[1].eos == 1 and p.env[1].limit_tension == 0.02
    assert p.projection_limiteur_id == 1 and p.ordre_projection == 2
    assert p.with_projection == 1 and p.cfl == 0.25
    assert p.deltat_init == 1e-5 and p.deltat_max == 0.01 and p.final_time == 0.2
    assert p.nb_bc == 6
    assert [p.bc[i].surface for i in range(6)] == [0, 3, 1, 4, 2, 5]
    assert p.time_history_period == 5


def test_lagrange_loop_disables_remap(tmp_path):
    text = open(ARC).read().replace("<timeloop>MahycoLoop</timeloop>", "<timeloop>MahycoLagrangeLoop</timeloop>")
    f = tmp_path / "lag.arc"
    f.write_text(text)
    p, info = read_arc(str(f))
    assert p.with_projection == 0


@pytest.mark.parametrize("snippet", ["<schema-csts>1</schema-csts>",
                                     "<coef-antiderive>0.1</coef-antiderive>"])
def test_unsupported_options_raise(tmp_path, snippet):
    text = open(ARC).read().replace("<pseudo-centree>0</pseudo-centree>", "<pseudo-centree>0</pseudo-centree>" + snippet)
    f = tmp_path / "u.arc"
    f.write_text(text)
    with pytest.raises(NotImplementedError):
        read_arc(str(f))


def test_params_roundtrip():
    p, _ = read_arc(ARC)
    q = params_from_dict(params_to_dict(p))
    assert bytes(p) == bytes(q)
