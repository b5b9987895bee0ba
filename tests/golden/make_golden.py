"""Extract golden fixtures from the reference's non-regression data.

Run with the root of a cea-hpc/MaHyCo checkout (the directory holding
NONREGRESSION/ and src/) as its first, required argument, optionally
followed by the cases to (re)make (all of CASES by default):

    python tests/golden/make_golden.py REFERENCE_ROOT [CASE ...]

For each case below it parses NONREGRESSION/<case>/Donnees.arc with
mahyco_b200.case.read_arc and stores the resulting parameters plus the
reference's EnvSummation time histories (output/courbes/gnuplot/<Var>_<Env>,
17 significant digits) in tests/golden/<case>.json.  The tests never read
the reference tree; they only read these JSON files.
"""
import ctypes
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from mahyco_b200.case import read_arc, params_to_dict  # noqa: E402
sys.path.insert(0, os.path.dirname(HERE))
import ensight_digest  # noqa: E402

# case -> extra oracle switches needed to reproduce how the reference ran it
CASES = {
    "CAS_2D_Lag_SodCaseX": {},
    "CAS_2D_Lag_SodCaseX_newton": {},
    "CAS_2D_Lag_BiSodCaseX": {"mpi_ranks": 4},
    "CAS_Lag_BiSodCaseX": {},
    "CAS_BiSodCaseX": {},
    # seq_pr test: 10 iterations, then a restart (launch_test.sh:25-38)
    "CAS_SodCaseX": {"restart_at": 10},
    "CAS_2D_Sedov": {},
    # run on 8 MPI ranks by the reference (src/CMakeLists.txt:193-208)
    "CAS_Sedov": {"mpi_ranks": 8},
    # third-order remap, run on 4 MPI ranks with 3 ghost layers
    # (src/CMakeLists.txt:164-189)
    "CAS_SodCaseX_ordre_3": {"mpi_ranks": 4},
    "CAS_SodCaseY_ordre_3": {"mpi_ranks": 4},
    "CAS_SodCaseZ_ordre_3": {"mpi_ranks": 4},
    "CAS_BiSodCaseX_ordre_3": {"mpi_ranks": 4},
    "CAS_BiSodCaseY_ordre_3": {"mpi_ranks": 4},
    "CAS_BiSodCaseZ_ordre_3": {"mpi_ranks": 4},
    # pente-borne fluxes, 4 MPI ranks with 2 ghost layers (the Z case has
    # no EnvSummation curves in the reference tree)
    "CAS_BiSodCaseX_pente_borne_minmod_debar_1": {"mpi_ranks": 4},
    "CAS_BiSodCaseX_pente_borne_minmod_debar_2": {"mpi_ranks": 4},
    "CAS_BiSodCaseX_pente_borne_superbee_debar_2": {"mpi_ranks": 4},
    "CAS_BiSodCaseY_pente_borne_minmod_debar_2": {"mpi_ranks": 4},
    "CAS_BiSodCaseY_pente_borne_superbee_debar_2": {"mpi_ranks": 4},
    # the other SOD directions and Lagrangian variants (src/CMakeLists.txt
    # TEST_NAMES and TEST_NAMES_PARA_4)
    "CAS_2D_Lag_SodCaseY": {"mpi_ranks": 4},
    "CAS_2D_Lag_SodCaseZ": {},
    "CAS_2D_Lag_BiSodCaseY": {"mpi_ranks": 4},
    "CAS_Lag_SodCaseX": {"mpi_ranks": 4},
    "CAS_Lag_SodCaseY": {},
    "CAS_Lag_SodCaseZ": {},
    "CAS_Lag_BiSodCaseY": {},
    "CAS_Lag_BiSodCaseZ": {"mpi_ranks": 4},
    "CAS_SodCaseY": {"mpi_ranks": 4},
    "CAS_SodCaseZ": {"mpi_ranks": 4},
    "CAS_BiSodCaseY": {"mpi_ranks": 4},
    "CAS_BiSodCaseZ": {"mpi_ranks": 4},
    # ONECELL init, LinearPressure / GeometricPressure surfaces, elasto
    # DefaultModel (EPP / YEPP), Mie-Gruneisen, explicit pressure; pressure
    # and energy grow from zero, so their first lines carry relative
    # differences up to 3e-10 that fall to 1e-13 as they grow
    "CAS_Compression_isotherme_ALU_monodimX": {"tol": 5e-10,
                                               # round-off residues (|value| <= 0.2 where XX reaches 1.7e8);
                                               # the plastic strain rate, (1 - coeff) Y / (3 mu coeff dt),
                                               # cancels in 1 - coeff and carries the 1e-10 state
                                               # differences into its 6th digit in 18 of 1000 cells
                                               "ensight_skip": ["StrainTensorYY/StrainTensorYY000001",
                                                                "StrainTensorXY/StrainTensorXY000001",
                                                                "PlasticDeformationVelocity/"
                                                                "PlasticDeformationVelocity000001"]},
    # per-axis Euler (is-euler-scheme Y), super-Gaussian energy deposit,
    # ONECELL init, Mie-Gruneisen; 200 000 equal cell masses averaged in one
    # running sum carry 3.7e-12 of rounding (the reference's four per-rank
    # sums 2.5e-13), hence the bound
    "CAS_plaque_demi_euler_Y_depot_Gaussian": {"mpi_ranks": 4, "tol": 1e-11},
    # sans-lagrange advection of the RIDER discs, Fictif equation of state
    # (src/CMakeLists.txt: the nsd of each Donnees.arc gives its ranks)
    "CAS_MonoRiderTx": {},
    "CAS_MonoRiderTy": {},
    "CAS_MonoRiderT45": {},
    "CAS_MonoRiderRotation": {},
    "CAS_MonoRiderDeformation": {},
    "CAS_RiderT45": {},
    "CAS_RiderTx": {"mpi_ranks": 8},
    "CAS_RiderTy": {"mpi_ranks": 8},
    "CAS_RiderRotation": {"mpi_ranks": 8},
    "CAS_RiderDeformation": {"mpi_ranks": 8},
    "CAS_RiderVortex": {"mpi_ranks": 8},
    "CAS_MonoRiderVortex": {"mpi_ranks": 8},
    "CAS_MonoRiderTy_pb_simple_superbee": {"mpi_ranks": 8},
    "CAS_MonoRiderTy_pb_mixte_superbee_vanleer": {"mpi_ranks": 8},
    "CAS_RiderVortexTimeReverse": {"mpi_ranks": 8},
    "CAS_MonoRiderVortexTimeReverse": {"mpi_ranks": 8},
    "CAS_RiderDeformationTimeReverse": {"mpi_ranks": 8},
    "CAS_MonoRiderDeformationTimeReverse": {"mpi_ranks": 8},
    # Gmsh grid (plaqueTaylor.msh, numbered column by column), EXTERNAL
    # init with a user velocity, Mie-Gruneisen, elasto-plastic, explicit
    # pressure, anti-hourglass.  The oracle's EnvSummation lines equal the
    # reference's bit for bit for the first 32 lines (320 iterations); then
    # the mean pressure drifts by at most 1.5e-5 relative (density 1.2e-9,
    # energy 6.8e-9); the reference's elasticity update reads an
    # uninitialised trace (elasto/DefaultModelService.cc:82, 96), which the
    # restatement takes as 0
    "CAS_2D_Lag_Taylor_elasto": {"exact_lines": 32, "time_tol": 3e-7,
                                 "tol_var": {"Pressure": 3e-5, "Density": 3e-9, "InternalEnergy": 2e-8},
                                 # the final state of the variables that the drift moves beyond 6 digits
                                 "ensight_skip": [f"{v}/{v}000001" for v in (
                                     "Pressure", "SoundSpeed", "Velocity", "StrainTensorXX", "StrainTensorYY",
                                     "StrainTensorXY", "PlasticDeformationVelocity")] +
                                 ["ensight.geo/ensight.geo000001"]},
    # the same bar and grid with NewHypoModel (the deviator's rate from the
    # left Cauchy-Green tensor of the accumulated deformation gradient): the
    # oracle's lines equal the reference's bit for bit for the first 9 lines
    # (90 iterations); then the time drifts by at most 2e-7 relative and the
    # mean pressure by 1.9e-3 (density 2e-9, energy 5e-9), like the
    # DefaultModel run above after its 32 exact lines
    "CAS_2D_Lag_Taylor_elasto_NeoHook": {"exact_lines": 9, "time_tol": 4e-7,
                                         "tol_var": {"Pressure": 2.5e-3, "Density": 4e-9, "InternalEnergy": 1e-8},
                                         "ensight_skip": [f"{v}/{v}000001" for v in (
                                             "Density", "InternalEnergy", "Pressure", "PseudoViscosity",
                                             "SoundSpeed", "Velocity", "StrainTensorXX", "StrainTensorYY",
                                             "StrainTensorXY", "PlasticDeformation",
                                             "PlasticDeformationVelocity")] +
                                         ["ensight.geo/ensight.geo000001"]},
    # Gmsh quarter annulus (noh.msh: 100 radial x 10 angular cells), EXTERNAL
    # init with the user velocity -x/|x|, OnFileVelocity on the outer radius,
    # 6020 Lagrangian iterations; with correctly rounded powers every line of
    # the reference's curves is reproduced bit for bit (glibc's pow moves
    # them by ulps from line 117 on)
    "CAS_2D_Lag_NOH": {"exact_lines_cr_pow": 602},
    # POINTTRIPLE init, three environments, 4 MPI ranks; the means of the
    # volumes, masses and energies stay within 7e-14 of the reference's, but
    # an environment's mean pressure can hang on a cell where it is nearly
    # absent, and one line of each run misses by 4e-11 (vanleer) or 6e-10
    # (pente-borne simple pente); the errors do not grow after it
    "CAS_bitriplepoint_minmod": {"mpi_ranks": 4, "tol_var": {"Pressure": 1e-10}},
    "CAS_MonoPointtriple_pb_sp_mixte_superbeeG_superbeeG": {"mpi_ranks": 4, "tol_var": {"Pressure": 2e-9}},
    # the same with the two-slope pente-borne fluxes is chaotic: two oracle
    # runs whose powers differ by an ulp part by 1e-2 after 2400 iterations,
    # so only the first 140 lines (1400 iterations) are kept, where the
    # 4-rank reference is still within 2e-13 (masses), 1e-11 (densities,
    # energies), 1e-8 (pressures)
    "CAS_MonoPointtriple_pb_mixte_superbeeG_superbeeG": {"mpi_ranks": 4, "lines": 140, "tol": 1e-10,
                                                          "tol_var": {"Pressure": 5e-8}},
}
# variables the Ensight writer of mahyco_b200.output produces
from mahyco_b200.output import ENSIGHT_VARS  # noqa: E402
VARS = ("CellMass", "Pressure", "Density", "InternalEnergy")


def main(ref_root, only=()):
    for case, extra in CASES.items():
        if only and case not in only:
            continue
        d = os.path.join(ref_root, "NONREGRESSION", case)
        p, info = read_arc(os.path.join(d, "Donnees.arc"))
        hist = {}
        for env in info["env_names"]:
            for v in VARS:
                fn = os.path.join(d, "output", "courbes", "gnuplot", f"{v}_{env}")
                if not os.path.exists(fn):
                    continue
                rows = [[float(x) for x in line.split()] for line in open(fn) if line.strip()]
                hist[f"{v}_{env}"] = rows[:extra["lines"]] if "lines" in extra else rows
        # digests of the reference's final Ensight files (6 significant
        # digits, round-off noise removed: tests/ensight_digest.py), compared
        # with the files mahyco_b200.output writes; a multi-rank reference
        # run writes only its first sub-domain, so none are kept for those
        dep = os.path.join(d, "output", "depouillement")
        digests = {}
        # (a mesh file's run is written in the file's numbering; a dataset
        # that post-processes variables the writer does not produce keeps the
        # digests of the geometry and of the variables it does)
        partial = not set(info["output_vars"]) <= ENSIGHT_VARS
        if extra.get("mpi_ranks", 1) == 1 and (not info["init_fields"] or "mesh_file" in info):
            for root, _, files in os.walk(dep):
                for fn in sorted(files):
                    full = os.path.join(root, fn)
                    rel = os.path.relpath(full, dep)
                    top = rel.split(os.sep)[0]
                    if partial and top not in ENSIGHT_VARS and top != "ensight.geo":
                        continue
                    if rel in extra.get("ensight_skip", ()):
                        continue
                    digests[rel] = ensight_digest.digest(full)
        out = {"case": case, "params": params_to_dict(p), "env_names": info["env_names"],
               "timeloop": info["timeloop"], "extra": extra, "time_history": hist,
               "output_vars": info["output_vars"], "save_init": info["save_init"], "ensight_sha256": digests}
        if info["init_fields"]:
            out["init_fields"] = info["init_fields"]
        if "mesh_file" in info:
            out["mesh_file"] = info["mesh_file"]
        with open(os.path.join(HERE, case + ".json"), "w") as f:
            json.dump(out, f, indent=0)
        print(case, {k: len(v) for k, v in hist.items()})


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_ROOT [CASE ...]")
    main(sys.argv[1], tuple(sys.argv[2:]))
