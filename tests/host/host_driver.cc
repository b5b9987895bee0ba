// host_driver.cc -- a C++ host that drives the hydro cycle through the C ABI
// alone (include/mahyco_b200.h), the way a MaHyCo-side module would: it
// fills the case options from the reference defaults, initialises the case,
// pushes part of its own state onto the device, runs iterations entry point
// by entry point in time-loop order (with the remap as its two service
// halves, appliRemap's sweeps then remapVariables, and the EOS services
// called per method), and reads the results back.
//
// usage: host_driver OUT_DIR NCYCLES
// writes OUT_DIR/params.bin (the mhc_case_params it used),
// OUT_DIR/uploaded_<Field>_<env>.bin (what it uploaded) and
// OUT_DIR/result_<Field>_<env>.bin (the fields after NCYCLES iterations),
// then prints one line "ok <iteration> <time> <deltat>".
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "mahyco_b200.h"

namespace {

#define CHECK(x)                                                                    \
  do {                                                                              \
    long long r_ = (long long)(x);                                                  \
    if (r_ < 0) {                                                                   \
      std::fprintf(stderr, "%s failed (%lld): %s\n", #x, r_, mhc_last_error());    \
      std::exit(1);                                                                 \
    }                                                                               \
  } while (0)

void write_bin(const std::string& path, const void* data, size_t bytes) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f || std::fwrite(data, 1, bytes, f) != bytes) {
    std::fprintf(stderr, "cannot write %s\n", path.c_str());
    std::exit(1);
  }
  std::fclose(f);
}

// 2D two-material Sod tube along x (CAS_2D_BiSodCaseX options), 60 x 8
// cells on [0,1] x [0,0.1], superbee, symmetry on every side
mhc_case_params bisod_case() {
  mhc_case_params p;
  mhc_case_params_default(&p);
  p.dim = 2;
  p.nx = 60; p.ny = 8; p.nz = 1;
  p.lx = 1.0; p.ly = 0.1; p.lz = 0.0;
  p.nb_env = 2;
  for (int e = 0; e < 2; ++e) p.env[e].specific_heat = 2.4;
  p.env[0].densite_initiale = 1.0;   p.env[0].pression_initiale = 1.0;
  p.env[1].densite_initiale = 0.125; p.env[1].pression_initiale = 0.1;
  p.cas_model = MHC_CASE_SOD;
  p.cas_test = MHC_TEST_BISOD_X;
  p.projection_limiteur_id = MHC_SUPERBEE;
  p.deltat_init = 1e-3;
  const int surf[4] = {MHC_XMIN, MHC_XMAX, MHC_YMIN, MHC_YMAX};
  const int kind[4] = {MHC_BC_VX, MHC_BC_VX, MHC_BC_VY, MHC_BC_VY};
  p.nb_bc = 4;
  for (int b = 0; b < 4; ++b) {
    p.bc[b].kind = kind[b];
    p.bc[b].surface = surf[b];
    p.bc[b].value = 0.0;
  }
  return p;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s OUT_DIR NCYCLES\n", argv[0]);
    return 2;
  }
  const std::string out = argv[1];
  const int ncycles = std::atoi(argv[2]);
  mhc_case_params p = bisod_case();
  write_bin(out + "/params.bin", &p, sizeof(p));
  const long long ncell = (long long)p.nx * p.ny;
  const long long nnode = (long long)(p.nx + 1) * (p.ny + 1);

  mhc_case* h = nullptr;
  CHECK(mhc_case_create(&p, &h));
  CHECK(mhc_hydro_start_init(h));

  // the host's own state: a warmer left environment (its internal energy
  // raised by a smooth bump along x), then the EOS services recompute
  // pressure and sound speed from it, per environment
  for (int env = 0; env < p.nb_env; ++env) {
    std::vector<double> e(ncell);
    CHECK(mhc_get_field(h, "InternalEnergy", env, e.data(), ncell));
    for (long long c = 0; c < ncell; ++c) {
      const double x = ((double)(c % p.nx) + 0.5) / p.nx;
      e[c] *= 1.0 + 0.25 * std::exp(-40.0 * (x - 0.3) * (x - 0.3));
    }
    CHECK(mhc_set_field(h, "InternalEnergy", env, e.data(), ncell));
    write_bin(out + "/uploaded_InternalEnergy_" + std::to_string(env) + ".bin", e.data(), ncell * 8);
    CHECK(mhc_eos_apply(h, env));
  }
  // a small initial velocity field
  std::vector<double> v(3 * nnode, 0.0);
  for (long long n = 0; n < nnode; ++n) {
    const long long i = n % (p.nx + 1);
    if (i > 0 && i < p.nx) v[3 * n] = 0.05 * std::sin(3.14159 * (double)i / p.nx);
  }
  CHECK(mhc_set_field(h, "Velocity", -1, v.data(), 3 * nnode));
  write_bin(out + "/uploaded_Velocity_-1.bin", v.data(), v.size() * 8);

  double gamma = 0.0;
  CHECK(mhc_eos_get_adiabatic_cst(h, 0, &gamma));
  if (gamma != 1.4) { std::fprintf(stderr, "adiabatic cst %g\n", gamma); return 1; }
  char euler[8];
  CHECK(mhc_remap_is_euler(h, euler, sizeof euler));
  const int nvars = 18 * p.nb_env;  // MahycoAnnexe.cc:65
  CHECK(mhc_remap_resize_remap_variables(h, nvars, p.nb_env));

  // the time loop, entry point by entry point (Mahyco.config:23-36)
  for (int it = 0; it < ncycles; ++it) {
    CHECK(mhc_save_values_at_n(h));
    CHECK(mhc_update_velocity(h));
    CHECK(mhc_apply_boundary_condition(h));
    CHECK(mhc_update_position(h));
    CHECK(mhc_compute_geometric_values(h));
    CHECK(mhc_update_density(h));
    CHECK(mhc_compute_artificial_viscosity(h));
    CHECK(mhc_update_elasticity_and_plasticity(h));
    CHECK(mhc_update_energy_and_pressure(h));
    // Remap: IRemap::appliRemap as its two halves
    CHECK(mhc_remap_synchronize_uremap(h));
    CHECK(mhc_remap_sweeps(h));
    CHECK(mhc_remap_variables(h, p.dim, 1, nvars, p.nb_env));
    CHECK(mhc_compute_delta_t(h));
  }
  const int status = mhc_synchronize(h);
  if (status != 0) { std::fprintf(stderr, "status %d\n", status); return 1; }

  const char* cell_fields[] = {"Density", "Pressure", "InternalEnergy", "SoundSpeed", "CellMass", "FracVol"};
  std::vector<double> buf(3 * nnode);
  for (const char* f : cell_fields) {
    for (int env = -1; env < p.nb_env; ++env) {
      if (env < 0 && std::string(f) == "FracVol") continue;
      const long long got = mhc_get_field(h, f, env, buf.data(), (long long)buf.size());
      CHECK(got);
      write_bin(out + "/result_" + f + "_" + std::to_string(env) + ".bin", buf.data(), got * 8);
    }
  }
  const long long got = mhc_get_field(h, "Velocity", -1, buf.data(), (long long)buf.size());
  CHECK(got);
  write_bin(out + "/result_Velocity_-1.bin", buf.data(), got * 8);
  double t = 0, dt = 0;
  long long iteration = 0;
  int st = 0;
  CHECK(mhc_get_scalars(h, &t, &dt, &iteration, &st));
  CHECK(mhc_case_destroy(h));
  std::printf("ok %lld %.17g %.17g\n", iteration, t, dt);
  return 0;
}
