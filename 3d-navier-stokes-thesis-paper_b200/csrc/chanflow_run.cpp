// chanflow_run.cpp -- the reference's DNS program (PFC/main_mpi.f90, the
// `mpiflow` executable) as a host program over the C ABI, on one GPU and
// without MPI: reads flow.dat (read_parms), sets up the grid and the
// wavenumbers (define_coordinates, define_parameters), makes the initial
// field (define_initial_field) and runs `timestep` with the reference's
// output cadence (PFC/main_mpi.f90:40-116): a VTK snapshot t_000.vtk before
// the loop when vel_out, WTIME every output_step steps, a VTK snapshot then
// when vel_out, the restart file newvel.out every save_step steps and once
// after the loop when save_vel, the l2 norm every l2_step steps, and for
// which_test 2 the mode's energy in fort.80 (PFC/pass2.f90:126-133).
//
//   chanflow_run flow.dat [--steps N] [--outdir DIR] [--device D] [--restart FILE]
//
// define_parameters' choices are kept: p_grad starts at -2/Re, or 0 with an
// x fringe (PFC/setup.f90:1384-1385) or for which_test 6; with read_vel = 1
// the initial field is the restart file (--restart, else savevel.out in the
// working directory, as read_velocity opens it, PFC/read_write.f90:34), and
// a missing file is an error; --restart with read_vel = 0 is refused.
// which_test 2, 5, 8 (the Orr-Sommerfeld mode of PFC/init_vel.f90:95-159)
// read the eigenfunction from efn.m in the working directory; their dt
// (cfh_read_flow_dat: 2 (2 pi / 0.24989154) / tend for tend >= 40,
// PFC/setup.f90:1386-1388) uses flow.dat's tend, so --steps runs a prefix of
// that run.
//
// The reference's RANDOM_NUMBER draws (initial field, jet forcing) are the
// library's seeded counter generator (cfh_rng_u01) with the flow.dat seed.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "chanflow.h"
#include "chanflow_host.h"

namespace {

void usage(FILE* f) {
  fprintf(f,
          "usage: chanflow_run flow.dat [--steps N] [--outdir DIR] [--device D] [--restart FILE]\n"
          "  runs the channel-flow DNS of flow.dat on one GPU (mpiflow's time loop):\n"
          "  --steps N      override tend\n"
          "  --outdir DIR   where t_###.vtk and restart files go (default .)\n"
          "  --device D     CUDA device (default 0)\n"
          "  --restart FILE initial field from a restart file (read_vel)\n");
}

int check(cfg_ctx* c, int r, const char* what) {
  if (r == CFG_OK) return 0;
  if (r == CFG_E_CFL) fprintf(stderr, "CFL IS TOO BIG\n");
  else if (r == CFG_E_DT) fprintf(stderr, "DT IS TOO BIG\n");
  else fprintf(stderr, "%s failed (%d): %s\n", what, r, c ? cfg_last_error(c) : "");
  return 1;
}

// the jet forcing parameters of define_parameters (PFC/setup.f90:1481-1491):
// amplitude, Strouhal number and two phases per (component, wall), and a
// random-walk increment of +-0.1 each
void jet_forcing_init(unsigned long long seed, double* jf, double* inc) {
  const double two_pi = 2.0 * std::acos(-1.0);
  for (int i = 0; i < 24; ++i) {
    const double u = cfh_rng_u01(seed, i, 0, 0, 5), v = cfh_rng_u01(seed, i, 0, 0, 6);
    const int kind = i / 6;   // (3,2,4) column-major: the last index is the slowest
    jf[i] = kind == 0 ? 0.01 + 0.06 * u : kind == 1 ? 0.1 + 0.6 * u : two_pi * u;
    inc[i] = v - 0.5 >= 0.0 ? 0.1 : -0.1;
  }
}

// ke(2,1) of rhs_solve (PFC/pass2.f90:113-117): the kinetic energy of Fourier
// column (kz 1, kx 2) of data1, |u|^2 + |w|^2 on the yh planes and |v|^2
// averaged onto them, integrated with dyh
double mode_energy(const cfh_grid* g, const double* data1) {
  const int nz = g->nz, nxh = g->nx / 2 + 1, n1 = g->ny + 1, ny = g->ny;
  auto at = [&](int j, int c, int k) { return data1[2 * (0 + (size_t)nz * (1 + (size_t)nxh * (j + (size_t)n1 * c))) + k]; };
  auto a2 = [&](int j, int c) { return at(j, c, 0) * at(j, c, 0) + at(j, c, 1) * at(j, c, 1); };
  double ke = 0.0;
  for (int j = 0; j < n1; ++j) {
    double t = a2(j, 0) + a2(j, 2);
    if (j == 0) t += a2(0, 1);
    else if (j < ny) {
      const double re = 0.5 * (at(j, 1, 0) + at(j - 1, 1, 0)), im = 0.5 * (at(j, 1, 1) + at(j - 1, 1, 1));
      t += re * re + im * im;
    } else t += a2(ny - 1, 1);
    ke += g->dyh[j] * t;
  }
  return ke;
}

}  // namespace

int main(int argc, char** argv) {
  const char* path = nullptr;
  const char* restart = nullptr;
  std::string outdir = ".";
  int steps = -1, device = 0;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "-h" || a == "--help") {
      usage(stdout);
      return 0;
    } else if (a == "--steps" && i + 1 < argc) {
      steps = atoi(argv[++i]);
    } else if (a == "--outdir" && i + 1 < argc) {
      outdir = argv[++i];
    } else if (a == "--device" && i + 1 < argc) {
      device = atoi(argv[++i]);
    } else if (a == "--restart" && i + 1 < argc) {
      restart = argv[++i];
    } else if (!a.empty() && a[0] != '-' && !path) {
      path = argv[i];
    } else {
      usage(stderr);
      return 2;
    }
  }
  if (!path) {
    usage(stderr);
    return 2;
  }
  // read_parms
  cfh_run run;
  cfh_run_defaults(&run);
  char err[256] = {0};
  if (cfh_read_flow_dat(path, &run, err, sizeof(err)) != 0) {
    fprintf(stderr, "%s: %s\n", path, err);
    return 1;
  }
  if (restart && run.read_vel != 1) {
    fprintf(stderr, "--restart given but %s has read_vel = %d (the initial field would not be read)\n", path,
            run.read_vel);
    return 2;
  }
  if (steps >= 0) run.tend = steps;
  if (run.output_step < 1) run.output_step = 1;
  if (run.save_step < 1) run.save_step = 1;
  if (run.l2_step < 1) run.l2_step = 1;
  // define_coordinates, define_parameters
  cfh_grid* g = cfh_grid_alloc(run.nx, run.ny, run.nz, run.nx2, run.nz2);
  if (!g || cfh_define_grid(g, run.lx, run.lz, run.stretch, run.uniform_grid) != 0) {
    fprintf(stderr, "grid set-up failed\n");
    cfh_grid_free(g);
    return 1;
  }
  cfg_params p{};
  p.nx = run.nx; p.ny = run.ny; p.nz = run.nz; p.nx2 = run.nx2; p.nz2 = run.nz2;
  p.re = run.re; p.lx = run.lx; p.lz = run.lz; p.beta = run.beta;
  p.dt = run.dt > 0.0 ? run.dt : 0.25 * run.lx / run.nx;   // PFC/setup.f90:1377
  p.cfl_max = 0.95;                                         // :1378
  p.fix_mass = run.fix_mass; p.dt_flag = run.dt_flag;
  p.ctrlu = run.ctrlu; p.ctrlw = run.ctrlw;
  p.precision = run.precision; p.device = device;
  cfg_grid cg{g->y, g->yh, g->hn, g->dh, g->dn, g->iu, g->dm, g->d2h, g->d2n, g->dyh, g->dy, g->kx, g->kz,
              nullptr, nullptr};
  cfg_ctx* c = nullptr;
  int r = cfg_create(&p, &cg, &c);
  if (r != CFG_OK) {
    fprintf(stderr, "cfg_create failed (%d)\n", r);
    cfh_grid_free(g);
    return 1;
  }
  int bad = 0;
  // p_grad = -2/Re, or 0 with an x fringe (PFC/setup.f90:1384-1385)
  if (run.xfringe == 1) bad = check(c, cfg_set_scalars(c, 0.0, p.dt, 0.0, nullptr), "cfg_set_scalars");
  // the fringe (init_buffer) and the crossflow jet (define_parameters)
  if (run.fringe_gain != 0.0 && (run.xfringe || run.zfringe)) {
    cfg_fringe f{run.fringe_gain, run.xfringe, run.zfringe, run.frac_xbuff, run.buff_xrise, run.buff_xfall,
                 run.frac_zbuff};
    bad = bad || check(c, cfg_init_buffer(c, &f), "cfg_init_buffer");
  }
  if (!bad && (run.crossflow == 1 || run.jet_mode != 0)) {
    cfg_jet j{};
    j.mode = run.jet_mode != 0 ? run.jet_mode : 1;
    j.xjet[0] = run.lx * run.xjet_bot; j.xjet[1] = run.lx * run.xjet_top;
    j.zjet[0] = run.lz * run.zjet_bot; j.zjet[1] = run.lz * run.zjet_top;
    j.jetmag[0] = run.jetmag_bot; j.jetmag[1] = run.jetmag_top;
    if (j.mode == 2) j.jetmag[0] = run.jet_peak;
    j.forcing[0] = run.forcing_bot; j.forcing[1] = run.forcing_top;
    j.for_freq[0] = run.for_freq_bot; j.for_freq[1] = run.for_freq_top;
    j.jet_diam = run.jet_diam;
    j.width = run.jet_width; j.freq = run.jet_freq;
    j.frac_xbuff = run.frac_xbuff;
    j.filter_jet_profile = run.filter_jet_profile;
    j.seed = run.seed;
    jet_forcing_init(run.seed, j.jet_forcing, j.jet_forcing_incr);
    bad = bad || check(c, cfg_set_jet(c, &j), "cfg_set_jet");
  }
  // define_initial_field
  if (!bad && run.read_vel == 1) {
    const char* file = restart ? restart : "savevel.out";
    bad = check(c, cfg_read_velocity(c, file), "cfg_read_velocity");
    if (bad) fprintf(stderr, "read_vel = 1: could not read the restart file %s\n", file);
  } else if (!bad) {
    const size_t n = (size_t)run.nz * (run.nx / 2 + 1) * (run.ny + 1) * 3 * 2;
    std::vector<double> d1(n, 0.0), d4(n / 3, 0.0);
    int ri = 0;
    if (run.which_test == 2 || run.which_test == 5 || run.which_test == 8) {
      // READ_EIGENFUNCTION: efn.m in the working directory
      std::vector<double> uin(4 * 65), u(2 * (run.ny + 1)), v(2 * (run.ny + 1));
      if (cfh_read_efn("efn.m", uin.data()) != 0) {
        fprintf(stderr, "which_test %d needs the eigenfunction file efn.m in the working directory\n",
                run.which_test);
        bad = 1;
      } else {
        cfh_interp_eigenfunction(g, uin.data(), u.data(), v.data());
        ri = cfh_initial_field_mode(g, run.which_test, run.disturb_ampl, run.beta, u.data(), v.data(), d1.data());
      }
    } else {
      ri = cfh_initial_field(g, run.which_test, run.seed, run.disturb_ampl, run.beta, d1.data());
    }
    if (!bad && ri != 0) {
      fprintf(stderr, "which_test %d is not supported\n", run.which_test);
      bad = 1;
    } else if (!bad) {
      bad = check(c, cfg_upload_state(c, d1.data(), nullptr, d4.data()), "cfg_upload_state");
      // which_test 6 (decaying vortices) runs without a mean pressure gradient
      if (!bad && run.which_test == 6) bad = check(c, cfg_set_scalars(c, 0.0, p.dt, 0.0, nullptr), "cfg_set_scalars");
    }
  }
  bad = bad || check(c, cfg_remove_initial_divergence(c), "cfg_remove_initial_divergence");
  bad = bad || check(c, cfg_compute_initial_pressure(c, 0), "cfg_compute_initial_pressure");
  double t_total = 0.0, dt = 0.0, p_grad = 0.0, l2 = 0.0, drag = 0.0;
  if (!bad) {
    cfg_get_scalars(c, &t_total, &dt, &p_grad, nullptr, nullptr);
    printf(" INITIAL DT = %.16e\n INITIAL TIME = %.16e\n", dt, t_total);
    bad = check(c, cfg_l2_norm(c, &l2, &drag), "cfg_l2_norm");
    if (!bad) printf(" l2 = %.10e  drag = %.10e\n", l2, drag);
    // the snapshot of the initial field (PFC/main_mpi.f90:42)
    if (!bad && run.vel_out == 1) bad = check(c, cfg_write_vtk(c, (outdir + "/t_000.vtk").c_str()), "cfg_write_vtk");
  }
  // the Orr-Sommerfeld run's record of the mode (fort.80, PFC/pass2.f90:126-133):
  // time, ke(2,1), p_grad and half log(ke)/time at every output step
  FILE* fort80 = nullptr;
  std::vector<double> d1out;
  if (!bad && run.which_test == 2 && run.read_vel == 0) {
    fort80 = fopen((outdir + "/fort.80").c_str(), "w");
    if (!fort80) {
      fprintf(stderr, "cannot write %s/fort.80\n", outdir.c_str());
      bad = 1;
    }
    d1out.resize((size_t)run.nz * (run.nx / 2 + 1) * (run.ny + 1) * 3 * 2);
  }
  // timestep
  auto t0 = std::chrono::steady_clock::now();
  for (int step = 1; step <= run.tend && !bad; ++step) {
    bad = check(c, cfg_timestep(c, 1), "cfg_timestep");
    if (bad) break;
    if (step % run.output_step == 0) {
      bad = check(c, cfg_synchronize(c), "cfg_synchronize");
      const auto t1 = std::chrono::steady_clock::now();
      printf("WTIME = %12.6f  OVER %6d  STEPS\n", std::chrono::duration<double>(t1 - t0).count(), run.output_step);
      fflush(stdout);
      if (!bad && run.vel_out == 1) {
        char name[64];
        snprintf(name, sizeof(name), "/t_%03d.vtk", step / run.output_step);
        bad = check(c, cfg_write_vtk(c, (outdir + name).c_str()), "cfg_write_vtk");
      }
      t0 = std::chrono::steady_clock::now();
    }
    if (!bad && run.save_vel == 1 && step % run.save_step == 0)
      bad = check(c, cfg_save_velocity(c, (outdir + "/newvel.out").c_str()), "cfg_save_velocity");
    if (!bad && fort80 && (step % run.output_step == 0 || step == run.tend)) {
      bad = check(c, cfg_download_state(c, d1out.data(), nullptr, nullptr), "cfg_download_state");
      if (!bad) {
        cfg_get_scalars(c, &t_total, &dt, &p_grad, nullptr, nullptr);
        const double ke = mode_energy(g, d1out.data());
        fprintf(fort80, "%10.3f%24.14E%24.14E%24.14E\n", t_total, ke, p_grad, 0.5 * std::log(ke + 1e-16) / t_total);
      }
    }
    if (!bad && step % run.l2_step == 0) {
      bad = check(c, cfg_status(c), "time step");
      if (!bad) bad = check(c, cfg_l2_norm(c, &l2, &drag), "cfg_l2_norm");
      if (!bad) printf(" step %d  l2 = %.10e  drag = %.10e\n", step, l2, drag);
    }
  }
  if (!bad) bad = check(c, cfg_status(c), "time step");
  // the final restart file (PFC/main_mpi.f90:46)
  if (!bad && run.save_vel == 1)
    bad = check(c, cfg_save_velocity(c, (outdir + "/newvel.out").c_str()), "cfg_save_velocity");
  if (!bad) bad = check(c, cfg_wait_io(c), "cfg_wait_io");
  if (!bad) {
    cfg_get_scalars(c, &t_total, &dt, &p_grad, nullptr, nullptr);
    printf(" FINAL TIME = %.16e  DT = %.16e  P_GRAD = %.16e\n", t_total, dt, p_grad);
  }
  if (fort80) fclose(fort80);
  cfg_destroy(c);
  cfh_grid_free(g);
  return bad ? 3 : 0;
}
