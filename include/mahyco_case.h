/*
 * mahyco_case.h -- plain-C description of one MaHyCo case (the subset of the
 * .arc dataset that the hydro cycle hot path reads).
 *
 * Field names and defaults follow the reference option descriptors:
 *   module options           src/Mahyco.axl:263-557
 *   RemapADI options         src/Remap/RemapADI.axl:162-210
 *   PerfectGas options       src/eos/perfectgas/PerfectGasEOS.axl:157-183
 *   StiffenedGas options     src/eos/stiffenedgas/StiffenedGasEOS.axl:158-184
 *   MieGruneisen options     src/eos/miegruneisen/MieGruneisenEOS.axl:157-219
 *   enums (BC kinds, limiter ids, case ids)  src/TypesMahyco.h:16-105
 *   cartesian mesh generator <meshgenerator><cartesian> block of the .arc files
 *
 * The struct is shared by the CUDA library (include/mahyco_b200.h) and by the
 * CPU oracle used by the tests; it contains no pointers, so it can be filled
 * from C, C++, Fortran or Python (ctypes) alike.  mhc_case_params_default()
 * (include/mahyco_b200.h) writes the reference defaults.
 */
#ifndef MAHYCO_CASE_H
#define MAHYCO_CASE_H

#ifdef __cplusplus
extern "C" {
#endif

#define MHC_MAX_ENV 4
#define MHC_MAX_BC 12
#define MHC_MAX_PTABLE 32

/* equation-of-state service kinds (<eos-model name="...">) */
enum mhc_eos_kind {
  MHC_EOS_PERFECT_GAS = 0,   /* PerfectGasEOSService.cc */
  MHC_EOS_STIFFENED_GAS = 1, /* StiffenedGasEOSService.cc */
  MHC_EOS_MIE_GRUNEISEN = 2, /* MieGruneisenEOSService.cc */
  MHC_EOS_FICTIF = 3         /* FictifEOSService.cc: the pressure a function of time only, sound
                                speed 1, internal energy reset to 0 (advection without Lagrange
                                phase, sans_lagrange) */
};

/* boundary-condition kinds, named after TypesMahyco::eBoundaryCondition
 * (TypesMahyco.h:16-32) and numbered in the order this library added them */
enum mhc_bc_kind {
  MHC_BC_VX = 0, MHC_BC_VY = 1, MHC_BC_VZ = 2,
  /* pressure applied as a node force on the surface (MahycoModule.cc:909-986) */
  MHC_BC_GEOMETRIC_PRESSURE = 3, MHC_BC_LINEAR_PRESSURE = 4,
  /* cell variables of the surface's cells (MahycoModule.cc:838-907): the
   * density (and cell mass, added to the node masses), an added internal
   * energy (flat or super-Gaussian in y, inside the x / y cutoffs), the
   * pressure */
  MHC_BC_DENSITY = 5, MHC_BC_ENERGY = 6, MHC_BC_SUPER_GAUSSIAN_ENERGY = 7, MHC_BC_PRESSURE = 8,
  /* pressure surfaces (MahycoModule.cc:952-970): the value times
   * exp(-(y dY)^power) exp(-(x dX)^power) at the node, 0 beyond |y| >
   * cutoffY; or times sqrt(1 - x^2/a2 - y^2/b2) at the boundary cell's
   * centre (a2 = dependanceX, b2 = dependanceY), 0 outside that ellipse */
  MHC_BC_SUPER_GAUSSIAN_PRESSURE = 9, MHC_BC_CONTACT_HERZ_PRESSURE = 10,
  /* OnFileVelocity ("OFV", MahycoModule.cc:796-798): the node's x and y
   * velocities set to -x / |X| and -y / |X| from its position X at the
   * start of the cycle (a unit velocity towards the origin); the value is
   * not used */
  MHC_BC_ON_FILE_VELOCITY = 11,
  /* OnFilePressure (MahycoModule.cc:987-1030): a pressure surface whose
   * value is the case's (time, pressure) table interpolated linearly at the
   * current time (0 before the first time and from the last time on), the
   * surface of every face node the length of the face
   * edge that starts at it (in 3D too), no time window; the value and
   * dependances are not used */
  MHC_BC_ON_FILE_PRESSURE = 12
};

/* energy deposits (TypesMahyco.h eEnergyDepot): constant, linear in
 * position and time, or super-Gaussian in x and y */
enum mhc_depot {
  MHC_DEPOT_NONE = 0, MHC_DEPOT_CONSTANT = 1, MHC_DEPOT_LINEAIRE = 2, MHC_DEPOT_SUPER_GAUSSIAN = 3
};

/* boundary surfaces built by MahycoModule::PrepareFaceGroup (MahycoAnnexe.cc:149-235) */
enum mhc_surface {
  MHC_XMIN = 0, MHC_YMIN = 1, MHC_ZMIN = 2, MHC_XMAX = 3, MHC_YMAX = 4, MHC_ZMAX = 5
};

/* remap limiter ids (TypesMahyco.h:96-105): classical (0-2) and the
 * generalised limiters of fluxLimiterG that use the cell widths (3-7) */
enum mhc_limiter {
  MHC_MINMOD = 0, MHC_SUPERBEE = 1, MHC_VANLEER = 2,
  MHC_MINMOD_G = 3, MHC_SUPERBEE_G = 4, MHC_VANLEER_G = 5, MHC_ARITHMETIC_G = 6, MHC_ULTRABEE_G = 7
};

/* case-initialisation services (<cas-model name="...">) */
enum mhc_case_model {
  MHC_CASE_SOD = 1,       /* casTest/SOD/SODService.cc */
  MHC_CASE_SEDOV = 2,     /* casTest/SEDOV/SEDOVService.cc */
  MHC_CASE_TWO_STATE = 3, /* explicit left/right states (seeded batch cases) */
  MHC_CASE_ONECELL = 4,   /* casTest/ONECELL/ONECELLService.cc: one uniform environment */
  MHC_CASE_BUBBLES = 5,   /* casTest/CHOCBULLE/CHOCBULLEService.cc: a lattice of bubbles of
                             environment 1 in environment 0 (mixed boundary cells) */
  MHC_CASE_RIDER = 6,     /* casTest/RIDER/RIDERService.cc: a disc advected by a prescribed
                             velocity field (cas_test 23-38) */
  MHC_CASE_EXTERNAL = 7,  /* casTest/EXTERNAL/EXTERNALService.cc (the default cas-model): the
                             dataset's <initialisation> block sets Materiau, Density and
                             Pressure per cell (mhc_case_set_initial_field; by default
                             environment 0 and its initial state everywhere), then
                             initUtilisateur sets the node velocities of every environment
                             with initialisation_utilisateur: its vitesse_initiale, or
                             -x/|x| when that is zero */
  MHC_CASE_TRIPLE_POINT = 8 /* casTest/POINTTRIPLE/POINTTRIPLEService.cc: three regions, x <= 0.01,
                               then y <= 0.015 or above, each holding environment 0, 1, 2
                               (BiTriplePoint, cas_test 12) or all environment 0 (MonoTriplePoint,
                               cas_test 2) with that environment's initial state; every node at
                               environment 0's initial velocity */
};

/* cas-test ids used by SOD, SEDOV, POINTTRIPLE and RIDER (TypesMahyco.h:44-94) */
enum mhc_cas_test {
  MHC_TEST_SEDOV = 1, MHC_TEST_MONO_TRIPLE_POINT = 2, MHC_TEST_SOD_X = 3, MHC_TEST_SOD_Y = 4, MHC_TEST_SOD_Z = 5,
  MHC_TEST_BISEDOV = 11, MHC_TEST_BI_TRIPLE_POINT = 12, MHC_TEST_BISOD_X = 13, MHC_TEST_BISOD_Y = 14,
  MHC_TEST_BISOD_Z = 15,
  /* RIDER: one environment (MonoRider*, 23-30) or a disc of environment 1 in
   * environment 0 (Rider*, 31-38); velocity a translation along x, y or the
   * diagonal, a rotation about (0.5, 0.5), a vortex or a deformation field */
  MHC_TEST_MONO_RIDER_TX = 23, MHC_TEST_MONO_RIDER_TY = 24, MHC_TEST_MONO_RIDER_T45 = 25,
  MHC_TEST_MONO_RIDER_ROTATION = 26, MHC_TEST_MONO_RIDER_VORTEX = 27, MHC_TEST_MONO_RIDER_DEFORMATION = 28,
  MHC_TEST_MONO_RIDER_VORTEX_REVERSE = 29, MHC_TEST_MONO_RIDER_DEFORMATION_REVERSE = 30,
  MHC_TEST_RIDER_TX = 31, MHC_TEST_RIDER_TY = 32, MHC_TEST_RIDER_T45 = 33, MHC_TEST_RIDER_ROTATION = 34,
  MHC_TEST_RIDER_VORTEX = 35, MHC_TEST_RIDER_DEFORMATION = 36, MHC_TEST_RIDER_VORTEX_REVERSE = 37,
  MHC_TEST_RIDER_DEFORMATION_REVERSE = 38,
  /* BiSodSph: the BiSod states inside and outside the sphere of radius 0.5
   * about the origin (SODService.cc:56-62) */
  MHC_TEST_BISOD_SPH = 39
};

/* longueur-caracteristique option values */
enum mhc_char_length {
  MHC_LENGTH_CUBE_ROOT_VOLUME = 0, /* "racine-cubique-volume" */
  MHC_LENGTH_OPPOSITE_FACES = 1,   /* "faces-opposees" */
  MHC_LENGTH_MONODIM_X = 2, MHC_LENGTH_MONODIM_Y = 3, MHC_LENGTH_MONODIM_Z = 4
};

/* is-euler-scheme option of RemapADI: Full (every axis back on the initial
 * grid), NON, or one axis X / Y / Z (only that axis is remapped and reset;
 * the other coordinates stay Lagrangian) */
enum mhc_euler_scheme {
  MHC_EULER_FULL = 0, MHC_EULER_NONE = 1, MHC_EULER_X = 2, MHC_EULER_Y = 3, MHC_EULER_Z = 4
};

typedef struct mhc_env_params {
  int eos;                       /* mhc_eos_kind */
  double adiabatic_cst;          /* adiabatic-cst (gamma) */
  double limit_tension;          /* limit-tension (p_inf for StiffenedGas) */
  double specific_heat;          /* specific-heat */
  double tension_damage_thresold;
  double density_damage_thresold;
  /* Mie-Gruneisen parameters */
  double rho0, s1, s2, s3, gamma0, a, c0, energie_ref, temperature_ref;
  /* pseudo-viscosity coefficients */
  double linear_pseudo_coeff, quadratic_pseudo_coeff;
  /* initial state */
  double densite_initiale, pression_initiale, energie_initiale, temperature_initiale;
  double vitesse_initiale[3];
  /* elasto-model: 0 NoModel, 1 DefaultModel (src/elasto/DefaultModelService.cc),
   * 2 NewHypoModel (src/elasto/NewHypoModelService.cc: the deviator's rate
   * from the left Cauchy-Green tensor of the accumulated deformation
   * gradient), each with the EPP shear modulus (elasto-mu-model elastic-cst)
   * and the YEPP yield strength (elasto-y-model limit-elastic);
   * ordre-rotation 1 or 2 */
  int elasto_model;
  int rotation_order;
  double shear_modulus;
  double yield_strength;
  /* energy-depot (MahycoModule.cc:1364-1417), added to the environment's
   * internal energy before the energy update: mhc_depot kind, value,
   * origine, dependanceX/Y/Z/T, cutoffX/Y, Tdebut, Tfin, power (exponent
   * of the super-Gaussian profile) */
  int depot_type;
  double depot_value;
  double depot_origin[3];
  double depot_dependance[4];
  double depot_cutoff[2];
  double depot_tdebut, depot_tfin;
  double depot_power;
  /* Fictif EOS (FictifEOS.axl): tdebut-pression, tfin-pression,
   * valeur-debut-pression, valeur-dependance-temps; the pressure is
   * p0 + dpdt t once t > tdebut, 0 once t > tfin */
  double fictif_tdebut, fictif_tfin, fictif_p0, fictif_dpdt;
  /* initialisation-utilisateur (Mahyco.axl): the EXTERNAL case model's
   * initUtilisateur runs for this environment */
  int initialisation_utilisateur;
} mhc_env_params;

typedef struct mhc_bc {
  int kind;     /* mhc_bc_kind */
  int surface;  /* mhc_surface */
  double value;
  double tdebut, tfin;
  double dependance[4];  /* LinearPressure: dependanceX, Y, Z, T; SuperGaussianEnergy: dependanceY */
  double cutoff[2];      /* Energy, SuperGaussianEnergy: cutoffX, cutoffY; SuperGaussianPressure: cutoffY */
  double power;          /* SuperGaussianPressure: the exponent (default 4) */
} mhc_bc;

typedef struct mhc_case_params {
  /* cartesian mesh generator */
  int dim;                  /* 2 or 3 */
  int nx, ny, nz;           /* cells per direction (nz ignored in 2D) */
  double origin[3];
  double lx, ly, lz;
  /* environments */
  int nb_env;
  mhc_env_params env[MHC_MAX_ENV];
  /* case model */
  int cas_model;            /* mhc_case_model */
  int cas_test;             /* mhc_cas_test */
  double sedov_energy;      /* total energy deposited by SEDOV (reference: 0.244816) */
  double interface_pos;     /* TWO_STATE: interface abscissa along interface_dir */
  int interface_dir;        /* TWO_STATE: 0=x 1=y 2=z */
  /* module options */
  int with_projection;
  int pseudo_centree;
  int with_newton;
  int pression_explicite;
  int deltat_constant;
  int calcul_vitson_max;
  int longueur_caracteristique; /* mhc_char_length */
  double cfl, deltat_init, deltat_min, deltat_max, final_time, threshold;
  double gravity[3];
  int nb_bc;
  mhc_bc bc[MHC_MAX_BC];
  /* RemapADI options */
  int ordre_projection;
  int projection_limiteur_id;
  int is_euler_scheme;
  double remap_threshold;
  /* EnvSummation period */
  int time_history_period;
  double coef_antiderive;   /* coef-antiderive: anti-hourglass velocity correction (Lagrange only) */
  int projection_simple_pente; /* projection-simple-pente: single-slope bound of the generalised limiters (pente-borne only) */
  int projection_pente_borne;  /* projection-pente-borne: fluxes integrated over the swept length */
  int projection_pente_borne_debar_fix; /* projection-pente-borne-debar-fix: 0, 1 (mean values) or 2 (cell values) */
  int projection_pente_borne_mixte;     /* projection-pente-borne-mixte: pure-neighbourhood fluxes */
  int projection_limiteur_pure_id;      /* projection-limiteur-pure-id: limiter of pure neighbourhoods */
  int conservation_energie_totale;      /* conservation-energie-totale: kinetic energy lost by the remap back to internal energy */
  /* BUBBLES case model (the bubble lattice of CHOCBULLE's cas-model
   * options): nombre-bulles-x/-y/-z, position-premiere-bulle,
   * deltax/deltay/deltaz-bulle, rayon-bulle.  A cell whose centre lies within
   * the radius of a bubble centre in the (x, y) plane belongs to the bubble
   * (environment 1; cylinders along z in 3D); it is mixed, with the bubble's
   * volume fraction (radius - dmin) / (dmax - dmin), when its nodes' (x, y)
   * distances to that centre range over [dmin, dmax] around the radius.
   * Environment 0 elsewhere. */
  int bubbles_n[3];
  double bubbles_first[3];
  double bubbles_delta[3];
  double bubbles_radius;
  /* sans-lagrange (Mahyco.axl): pure advection.  The node velocities are
   * prescribed (those of the initialisation, times cos(Pi t parameter) with
   * the RIDER reverse option), only nodes shared by exactly four cells move,
   * the density, pseudo-viscosity and energy updates are skipped, the time
   * step stays deltat_init, and the remap projects the cells only (no dual
   * projection: the velocities are not remapped). */
  int sans_lagrange;
  /* RIDER case model options (RIDER.axl): reverse-option, parametre,
   * rayon-bulle, densite-interieure-initiale-lineaire */
  int rider_reverse;
  double rider_parameter;
  double rider_radius;
  int rider_linear_density;
  /* schema-csts (Mahyco.axl:396-399), with the remap: the velocities go
   * back to n-1/2 before the node pass (updateVelocityBackward) and forward
   * to n+1 before the remap (updateVelocityForward), the ideal-gas energy
   * update takes the work of the forces at n and n+1 through the corner
   * normals, and the remap's face velocities are the mean of those at n and
   * n+1 */
  int schema_csts;
  /* order of the cells in the reference's numbering, which fixes the order
   * of its sums over cells (node forces and masses, the anti-hourglass
   * correction, the time history): 0 x-fastest (the cartesian generator),
   * 1 y-fastest (the 2D Gmsh quadrangle grids of the datasets, whose
   * elements run column by column) */
  int mesh_cell_order;
  /* the (time, pressure) table of OnFilePressure, which the reference reads
   * from Pression.data at init (lireFichierCDL, MahycoAnnexe.cc:242-269):
   * pressure_table_n pairs in the file's order */
  int pressure_table_n;
  double pressure_table_t[MHC_MAX_PTABLE];
  double pressure_table_p[MHC_MAX_PTABLE];
} mhc_case_params;

#ifdef __cplusplus
}
#endif
#endif
