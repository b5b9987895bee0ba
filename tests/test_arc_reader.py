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


def test_schema_csts_is_read(tmp_path):
    text = open(ARC).read().replace("<pseudo-centree>0</pseudo-centree>",
                                    "<pseudo-centree>0</pseudo-centree><schema-csts>1</schema-csts>")
    f = tmp_path / "u.arc"
    f.write_text(text)
    p, _ = read_arc(str(f))
    assert p.schema_csts == 1


def test_params_roundtrip():
    p, _ = read_arc(ARC)
    q = params_from_dict(params_to_dict(p))
    assert bytes(p) == bytes(q)


def test_anti_hourglass_and_elasto_options(tmp_path):
    """coef-antiderive and the DefaultModel/EPP/YEPP elasto block are read
    (CAS_2D_Lag_Taylor_elasto style); other elasto models are refused."""
    text = open(ARC).read().replace("<pseudo-centree>0</pseudo-centree>",
                                    "<pseudo-centree>0</pseudo-centree><coef-antiderive>0.01</coef-antiderive>")
    f = tmp_path / "h.arc"
    f.write_text(text)
    p, _ = read_arc(str(f))
    assert p.coef_antiderive == 0.01
    el = ('<elasto-model name="DefaultModel"><ordre-rotation>2</ordre-rotation>'
          '<elasto-mu-model name="EPP"><elastic-cst>2.6e10</elastic-cst></elasto-mu-model>'
          '<elasto-y-model name="YEPP"><limit-elastic>3.e8</limit-elastic></elasto-y-model></elasto-model>')
    src = open(ARC).read()
    i = src.index("</environment>")
    f2 = tmp_path / "e.arc"
    f2.write_text(src[:i] + el + src[i:])
    p2, _ = read_arc(str(f2))
    assert (p2.env[0].elasto_model, p2.env[0].rotation_order) == (1, 2)
    assert (p2.env[0].shear_modulus, p2.env[0].yield_strength) == (2.6e10, 3.e8)
    f3 = tmp_path / "n.arc"
    f3.write_text(src[:i] + el.replace("DefaultModel", "NewHypoModel") + src[i:])
    p3, _ = read_arc(str(f3))
    assert (p3.env[0].elasto_model, p3.env[0].rotation_order) == (2, 2)
    f4 = tmp_path / "m.arc"
    f4.write_text(src[:i] + el.replace('"EPP"', '"SCG"') + src[i:])
    with pytest.raises(NotImplementedError):
        read_arc(str(f4))


def test_remap_order_and_generalised_limiter_options(tmp_path):
    """ordre-projection 3, the generalised limiters (ids 3-7), the
    pente-borne options, projection-simple-pente and
    conservation-energie-totale are read."""
    text = open(ARC).read().replace("<ordre-projection>2</ordre-projection>",
                                    "<ordre-projection>3</ordre-projection>").replace(
        "<projection-limiteur-id>1</projection-limiteur-id>",
        "<projection-limiteur-id>5</projection-limiteur-id>"
        "<projection-simple-pente>true</projection-simple-pente>")
    assert text != open(ARC).read()
    f = tmp_path / "o3.arc"
    f.write_text(text)
    p, _ = read_arc(str(f))
    assert (p.ordre_projection, p.projection_limiteur_id, p.projection_simple_pente) == (3, 5, 1)
    g = tmp_path / "pb.arc"
    g.write_text(text.replace("<ordre-projection>3</ordre-projection>",
                              "<projection-pente-borne>true</projection-pente-borne>"
                              "<projection-pente-borne-debar-fix>1</projection-pente-borne-debar-fix>"
                              "<projection-pente-borne-mixte>true</projection-pente-borne-mixte>"
                              "<projection-limiteur-pure-id>1</projection-limiteur-pure-id>"))
    q, _ = read_arc(str(g))
    assert (q.projection_pente_borne, q.projection_pente_borne_debar_fix, q.projection_pente_borne_mixte,
            q.projection_limiteur_pure_id, q.ordre_projection) == (1, 1, 1, 1, 2)
    r = tmp_path / "cet.arc"
    r.write_text(text.replace("<ordre-projection>3</ordre-projection>",
                              "<conservation-energie-totale>true</conservation-energie-totale>"))
    assert read_arc(str(r))[0].conservation_energie_totale == 1


def test_gnuplot_writer_format(tmp_path):
    """EnvSummation curves in the reference's layout: <Var>_<Env>, one
    'time value' line, 17 significant digits; absent environments skipped."""
    import numpy as np
    from mahyco_b200.output import write_gnuplot
    rows = np.array([[1.2577892535548833e-04, 2.5, 1.0, 0.9999974710589157, 3.0, 1.0, 0., 0., 0., 0., 0.]])
    files = write_gnuplot(str(tmp_path), ["ZG", "ZD"], rows)
    assert sorted(os.path.basename(f) for f in files) == ["CellMass_ZG", "Density_ZG", "InternalEnergy_ZG",
                                                          "Pressure_ZG"]
    assert open(tmp_path / "courbes" / "gnuplot" / "Density_ZG").read() == \
        "1.2577892535548833E-04 9.9999747105891568E-01\n"


def test_energy_deposit_options(tmp_path):
    """<energy-depot> of an environment (Mahyco.axl:335-380): constant,
    linear and super-Gaussian deposits with their power (default 4)."""
    dep = ("<energy-depot><type>DepotLineaire</type><valeur-source-energie>3.5e3</valeur-source-energie>"
           "<origine>0.1 0.2 0.</origine><dependanceX>2.</dependanceX><dependanceT>5.</dependanceT>"
           "<cutoffY>0.5</cutoffY><Tdebut>1e-3</Tdebut><Tfin>2e-3</Tfin></energy-depot>")
    text = open(ARC).read().replace("</environment>", dep + "</environment>", 1)
    f = tmp_path / "d.arc"
    f.write_text(text)
    p, _ = read_arc(str(f))
    e = p.env[0]
    assert (e.depot_type, e.depot_value, list(e.depot_origin)) == (2, 3.5e3, [0.1, 0.2, 0.0])
    assert list(e.depot_dependance) == [2.0, 0.0, 0.0, 5.0] and list(e.depot_cutoff) == [1000.0, 0.5]
    assert (e.depot_tdebut, e.depot_tfin, p.env[1].depot_type) == (1e-3, 2e-3, 0)
    assert e.depot_power == 4.0
    g = tmp_path / "g.arc"
    g.write_text(text.replace("DepotLineaire", "DepotSuperGaussian").replace("<Tfin>", "<power>8.</power><Tfin>"))
    e = read_arc(str(g))[0].env[0]
    assert (e.depot_type, e.depot_power) == (3, 8.0)


def test_per_axis_euler_scheme(tmp_path):
    """<is-euler-scheme> of RemapADI (RemapADI.axl:169): Full, X, Y, Z; NON
    (a remap that never returns to the grid) is refused."""
    text = open(ARC).read()
    assert read_arc(ARC)[0].is_euler_scheme == 0
    for name, v in (("X", 2), ("Y", 3), ("Z", 4), ("Full", 0)):
        f = tmp_path / f"e{name}.arc"
        f.write_text(text.replace("</ordre-projection>",
                                  f"</ordre-projection><is-euler-scheme>{name}</is-euler-scheme>", 1))
        assert read_arc(str(f))[0].is_euler_scheme == v
    f = tmp_path / "non.arc"
    f.write_text(text.replace("</ordre-projection>", "</ordre-projection><is-euler-scheme>NON</is-euler-scheme>", 1))
    with pytest.raises(NotImplementedError):
        read_arc(str(f))


def test_pressure_surfaces_and_onecell(tmp_path):
    """LinearPressure / GeometricPressure surfaces with their time window
    and linear dependences, the ONECELL init and the output-history-period
    that thins the EnvSummation lines (here lcm(10, 500) = 500)."""
    text = open(ARC).read().replace('<cas-model name="SOD">', '<cas-model name="ONECELL">').replace(
        "<cas-test>13</cas-test>", "<cas-test>0</cas-test>").replace(
        "<final-time>", "<boundary-condition><surface>XMAX</surface><type>LinearPressure</type><value>1.</value>"
        "<dependanceT>3e17</dependanceT><Tfin>1e-7</Tfin></boundary-condition>"
        "<boundary-condition><surface>XMIN</surface><type>GeometricPressure</type><value>30e9</value>"
        "<Tdebut>1e-7</Tdebut></boundary-condition><final-time>", 1).replace(
        "<mesh", "<arcane-post-processing><output-history-period>500</output-history-period>"
        "</arcane-post-processing><mesh", 1)
    f = tmp_path / "p.arc"
    f.write_text(text)
    p, _ = read_arc(str(f))
    assert p.cas_model == 4 and p.time_history_period == 500
    kinds = [(p.bc[i].kind, p.bc[i].surface, p.bc[i].value, p.bc[i].tdebut, p.bc[i].tfin, list(p.bc[i].dependance))
             for i in range(p.nb_bc)]
    assert (4, 3, 1.0, 0.0, 1e-7, [0.0, 0.0, 0.0, 3e17]) in kinds
    assert (3, 0, 30e9, 1e-7, 1000.0, [0.0, 0.0, 0.0, 0.0]) in kinds


def test_on_file_boundary_conditions(tmp_path):
    """OFV (OnFileVelocity) and OnFilePressure (Mahyco.axl:498, 505); the
    pressure table comes from Pression.data beside the dataset, whatever
    the fichier option names, read two reals at a time (MahycoAnnexe.cc:
    242-269); without that file the table stays empty."""
    bcs = ("<boundary-condition><surface>XMAX</surface><type>OFV</type><value>1.</value></boundary-condition>"
           "<boundary-condition><surface>XMIN</surface><type>OnFilePressure</type><value>-1.</value>"
           "<fichier>other.data</fichier></boundary-condition>")
    text = open(ARC).read().replace("<final-time>", bcs + "<final-time>", 1)
    f = tmp_path / "o.arc"
    f.write_text(text)
    p, _ = read_arc(str(f))
    got = [(p.bc[i].kind, p.bc[i].surface) for i in range(p.nb_bc) if p.bc[i].kind >= 11]
    assert got == [(11, 3), (12, 0)]
    assert p.pressure_table_n == 0
    (tmp_path / "Pression.data").write_text("0. 0.\n1.00e-11 10.0e9\n9.00e-9  10.0e9\n9.01e-9  0.\n")
    p, _ = read_arc(str(f))
    assert p.pressure_table_n == 4
    assert list(p.pressure_table_t[:4]) == [0.0, 1e-11, 9e-9, 9.01e-9]
    assert list(p.pressure_table_p[:4]) == [0.0, 1e10, 1e10, 0.0]


def test_cell_variable_boundary_conditions(tmp_path):
    """Density / Energy / SuperGaussianEnergy / Pressure conditions
    (Mahyco.axl:490-535) with their cutoffs (default 1000)."""
    bcs = ("<boundary-condition><surface>XMIN</surface><type>Density</type><value>2.</value></boundary-condition>"
           "<boundary-condition><surface>YMAX</surface><type>SuperGaussianEnergy</type><value>3.</value>"
           "<dependanceY>5.</dependanceY><cutoffY>0.25</cutoffY></boundary-condition>"
           "<boundary-condition><surface>XMAX</surface><type>Pressure</type><value>4.</value>"
           "<Tdebut>1e-3</Tdebut></boundary-condition>")
    text = open(ARC).read().replace("<final-time>", bcs + "<final-time>", 1)
    f = tmp_path / "c.arc"
    f.write_text(text)
    p, _ = read_arc(str(f))
    got = [(p.bc[i].kind, p.bc[i].surface, p.bc[i].value, p.bc[i].tdebut, list(p.bc[i].cutoff))
           for i in range(p.nb_bc) if p.bc[i].kind >= 5]
    assert got == [(5, 0, 2.0, 0.0, [1000.0, 1000.0]), (7, 4, 3.0, 0.0, [1000.0, 0.25]),
                   (8, 3, 4.0, 1e-3, [1000.0, 1000.0])]
    assert [p.bc[i].dependance[1] for i in range(p.nb_bc) if p.bc[i].kind == 7] == [5.0]


def test_read_chocbulle_lattice(tmp_path):
    """The bubble lattice options of CHOCBULLE's cas-model
    (src/casTest/CHOCBULLE/CHOCBULLE.axl:180-202) fill the BUBBLES case."""
    from mahyco_b200.case import CASE_BUBBLES
    text = open(ARC).read()
    start, end = text.index("<cas-model"), text.index("</cas-model>") + len("</cas-model>")
    block = ("<cas-model name=\"CHOCBULLE\"><cas-test>47</cas-test>"
             "<nombre-bulles-x>2</nombre-bulles-x><nombre-bulles-y>3</nombre-bulles-y>"
             "<position-premiere-bulle>0.3 0.1 0.0</position-premiere-bulle>"
             "<deltax-bulle>0.1</deltax-bulle><deltay-bulle>0.05</deltay-bulle>"
             "<rayon-bulle>0.02</rayon-bulle><nombre-bulles-aleatoires>0</nombre-bulles-aleatoires></cas-model>")
    f = tmp_path / "bulles.arc"
    f.write_text(text[:start] + block + text[end:])
    p, _ = read_arc(str(f))
    assert p.cas_model == CASE_BUBBLES and p.cas_test == 47
    assert list(p.bubbles_n) == [2, 3, 1] and list(p.bubbles_first) == [0.3, 0.1, 0.0]
    assert list(p.bubbles_delta) == [0.1, 0.05, 0.0] and p.bubbles_radius == 0.02
    f.write_text(text[:start] + block.replace("<nombre-bulles-aleatoires>0", "<nombre-bulles-aleatoires>4") + text[end:])
    with pytest.raises(NotImplementedError):
        read_arc(str(f))


def test_rider_fictif_sans_lagrange_options(tmp_path):
    """A RIDER cas-model (src/casTest/RIDER/RIDER.axl:145-166), Fictif
    equations of state (src/eos/fictif/FictifEOS.axl:184-196),
    sans-lagrange and save-init (CAS_*Rider* style)."""
    from mahyco_b200.case import CASE_RIDER, EOS_FICTIF
    text = open(ARC).read()
    start, end = text.index("<cas-model"), text.index("</cas-model>") + len("</cas-model>")
    block = ("<cas-model name=\"RIDER\"><cas-test>38</cas-test><reverse-option>true</reverse-option>"
             "<parametre>1.</parametre><rayon-bulle>0.2</rayon-bulle></cas-model>")
    text = text[:start] + block + text[end:]
    text = text.replace("<pseudo-centree>0</pseudo-centree>",
                        "<pseudo-centree>0</pseudo-centree><sans-lagrange>true</sans-lagrange>")
    text = text.replace("</arcane>", "</arcane><arcane-post-processing><save-init>true</save-init>"
                                      "</arcane-post-processing>", 1)
    fictif = ("<eos-model name=\"Fictif\"><tdebut-pression>0.1</tdebut-pression><tfin-pression>10</tfin-pression>"
              "<valeur-debut-pression>2.</valeur-debut-pression><valeur-dependance-temps>3.</valeur-dependance-temps>")
    for name in ("PerfectGas", "StiffenedGas"):
        text = text.replace(f"<eos-model name=\"{name}\">", fictif)
    f = tmp_path / "rider.arc"
    f.write_text(text)
    p, info = read_arc(str(f))
    assert p.cas_model == CASE_RIDER and p.cas_test == 38 and p.sans_lagrange == 1
    assert p.rider_reverse == 1 and p.rider_parameter == 1.0 and p.rider_radius == 0.2 and p.rider_linear_density == 0
    assert info["save_init"] is True
    for e in range(p.nb_env):
        o = p.env[e]
        assert o.eos == EOS_FICTIF
        assert (o.fictif_tdebut, o.fictif_tfin, o.fictif_p0, o.fictif_dpdt) == (0.1, 10.0, 2.0, 3.0)
