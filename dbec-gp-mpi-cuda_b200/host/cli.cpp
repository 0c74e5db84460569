// cli.cpp -- main programs of imag3d-mpicuda and real3d-mpicuda over the C ABI.
//
// Mirrors main() and readpar() of src/imag3d-mpicuda/imag3d-mpicuda.cu
// (:29-829) and src/real3d-mpicuda/real3d-mpicuda.cu (:29-883): the same
// required keys and messages, the same phase structure (NSTP ramp, NPAS,
// quench, NRUN), the same fprintf formats and the same output files.  MPI is
// gone: the header still prints MPI_NUM_PROCS = 1, and the MPI-IO writes
// become pwrite() on files opened without truncation, as MPI_File_open with
// MPI_MODE_WRONLY | MPI_MODE_CREATE does.
#include "cli.h"

#include <fcntl.h>
#include <unistd.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "cfg.h"
#include "gpe.h"

namespace gpecli {

namespace {

const double kPi = 3.14159265358979;             // imag3d-mpicuda.cu:69
const double kBohrRadius = 5.2917720859e-11;     // imag3d-mpicuda.cuh:46

struct Par {
   int opt = 0;
   long Na = 0;
   double g0 = 0, gd0 = 0, aho = 0, as = 0, add = 0;
   double gpar = 1, gdpar = 1;
   long Nx = 0, Ny = 0, Nz = 0;
   double dx = 0, dy = 0, dz = 0, dt = 0;
   double vgamma = 0, vnu = 0, vlambda = 0;
   long Nstp = 0, Npas = 0, Nrun = 0;
   double cutoff = 0;
   const char *output = nullptr, *rmsout = nullptr, *dynaout = nullptr;
   const char *initout = nullptr, *nstpout = nullptr, *npasout = nullptr, *nrunout = nullptr;
   long outstpx = 1, outstpy = 1, outstpz = 1, outstpt = 0;
   int device = -1;
   int potmem = 2;
};

[[noreturn]] void die(const char *msg) {
   std::fputs(msg, stderr);
   std::exit(EXIT_FAILURE);
}

const char *need(const char *key, const char *msg) {
   const char *v = cfg_read(key);
   if (!v) die(msg);
   return v;
}

// readpar (imag3d-mpicuda.cu:650-829, real3d-mpicuda.cu:675-883).
void readpar(int mode, Par &p) {
   const bool real = mode == 1;
   p.opt = (int) std::atol(need("OPTION", "OPTION is not defined in the configuration file\n"));
   p.Na = std::atol(need("NATOMS", "NATOMS is not defined in the configuration file.\n"));
   const char *t;
   if ((t = cfg_read("G0")) == nullptr) {
      p.aho = std::atof(need("AHO", "AHO is not defined in the configuration file.\n"));
      p.as = std::atof(need("AS", "AS is not defined in the configuration file.\n"));
      p.g0 = 4. * kPi * p.as * p.Na * kBohrRadius / p.aho;
   } else {
      p.g0 = std::atof(t);
   }
   if (real) p.gpar = std::atof(need("GPAR", "GPAR is not defined in the configuration file.\n"));
   if ((t = cfg_read("GDD0")) == nullptr) {
      p.aho = std::atof(need("AHO", "AHO is not defined in the configuration file.\n"));
      p.add = std::atof(need("ADD", "ADD is not defined in the configuration file.\n"));
      p.gd0 = 3. * p.add * p.Na * kBohrRadius / p.aho;
   } else {
      p.gd0 = std::atof(t);
   }
   if (real) p.gdpar = std::atof(need("GDDPAR", "GDDPAR is not defined in the configuration file.\n"));
   p.Nx = std::atol(need("NX", "NX is not defined in the configuration file.\n"));
   p.Ny = std::atol(need("NY", "NY is not defined in the configuration file.\n"));
   p.Nz = std::atol(need("NZ", "Nz is not defined in the configuration file.\n"));
   p.dx = std::atof(need("DX", "DX is not defined in the configuration file.\n"));
   p.dy = std::atof(need("DY", "DY is not defined in the configuration file.\n"));
   p.dz = std::atof(need("DZ", "DZ is not defined in the configuration file.\n"));
   p.dt = std::atof(need("DT", "DT is not defined in the configuration file.\n"));
   p.vgamma = std::atof(need("GAMMA", "GAMMA is not defined in the configuration file.\n"));
   p.vnu = std::atof(need("NU", "NU is not defined in the configuration file.\n"));
   p.vlambda = std::atof(need("LAMBDA", "LAMBDA is not defined in the configuration file.\n"));
   p.Nstp = std::atol(need("NSTP", "NSTP is not defined in the configuration file.\n"));
   p.Npas = std::atol(need("NPAS", "NPAS is not defined in the configuration file.\n"));
   p.Nrun = std::atol(need("NRUN", "NRUN is not defined in the configuration file.\n"));
   p.cutoff = std::atof(need("CUTOFF", "CUTOFF is not defined in the configuration file.\n"));
   p.output = cfg_read("OUTPUT");
   p.rmsout = cfg_read("RMSOUT");
   if (real) p.dynaout = cfg_read("DYNAOUT");
   p.initout = cfg_read("INITOUT");
   p.nstpout = cfg_read("NSTPOUT");
   p.npasout = cfg_read("NPASOUT");
   p.nrunout = cfg_read("NRUNOUT");
   if (p.initout || p.nstpout || p.npasout || p.nrunout) {
      p.outstpx = std::atol(need("OUTSTPX", "OUTSTPX is not defined in the configuration file.\n"));
      p.outstpy = std::atol(need("OUTSTPY", "OUTSTPY is not defined in the configuration file.\n"));
      p.outstpz = std::atol(need("OUTSTPZ", "OUTSTPZ is not defined in the configuration file.\n"));
   }
   if (real && p.rmsout) p.outstpt = std::atol(need("OUTSTPT", "OUTSTPT is not defined in the configuration file.\n"));
   if (real && p.dynaout) p.outstpt = std::atol(need("OUTSTPT", "OUTSTPT is not defined in the configuration file.\n"));
   p.device = (t = cfg_read("DEVICE")) ? std::atoi(t) : -1;
   if ((t = cfg_read("POTMEM")) != nullptr) {
      // POTMEM selected where the reference kept V and Udd (host-mapped,
      // re-uploaded or resident); the tables here are always resident.
      p.potmem = std::atoi(t);
      if (p.potmem < 0 || p.potmem > 2) die("POTMEM can be 0, 1 or 2.\n");
   }
}

void check(gpe_status st, const char *what) {
   if (st != GPE_OK) {
      std::fprintf(stderr, "%s failed: %s\n", what, gpe_last_error());
      std::exit(EXIT_FAILURE);
   }
}

// MPI_File_open(MPI_MODE_WRONLY | MPI_MODE_CREATE) + write_at: no truncation.
void write_file(const std::string &name, const double *v, size_t n) {
   int fd = ::open(name.c_str(), O_WRONLY | O_CREAT, 0644);
   if (fd < 0) {
      std::fprintf(stderr, "cannot open %s for writing\n", name.c_str());
      std::exit(EXIT_FAILURE);
   }
   const char *p = (const char *) v;
   size_t left = n * sizeof(double);
   off_t off = 0;
   while (left > 0) {
      ssize_t w = ::pwrite(fd, p, left, off);
      if (w <= 0) {
         std::fprintf(stderr, "write to %s failed\n", name.c_str());
         std::exit(EXIT_FAILURE);
      }
      p += w; off += w; left -= (size_t) w;
   }
   ::close(fd);
}

// outdenxyz, outdenx/y/z, outdenxy/xz/yz, outpsi2xy/xz/yz of one phase
// (imag3d-mpicuda.cu:253-299 for INITOUT; the same list after each phase).
void write_densities(gpe_solver *s, const Par &p, const char *prefix, bool z_as_txt) {
   const long n3 = p.Nx * p.Ny * p.Nz;
   std::vector<double> buf((size_t) (n3 + 3 * (p.Nx * p.Ny + p.Nx * p.Nz + p.Ny * p.Nz) + 16));
   long cnt = 0;
   std::string pre(prefix);
   // raw 3D density: rows of Nz/OUTSTPZ samples (outdenxyz, imag:2355-2381)
   check(gpe_density(s, GPE_DEN_3D, p.outstpx, p.outstpy, p.outstpz, buf.data(), (long) buf.size(), &cnt), "density");
   {
      const long nk = (p.Nz + p.outstpz - 1) / p.outstpz, row = p.Nz / p.outstpz;
      std::vector<double> o;
      for (long r = 0; r < cnt / nk; r++) o.insert(o.end(), buf.begin() + r * nk, buf.begin() + r * nk + row);
      write_file(pre + ".bin", o.data(), o.size());
   }
   struct Item { int kind; const char *suffix; };
   const Item items[] = {{GPE_DEN_1D_X, "1d_x.bin"},  {GPE_DEN_1D_Y, "1d_y.bin"},   {GPE_DEN_1D_Z, "1d_z.bin"},
                         {GPE_DEN_2D_XY, "2d_xy.bin"}, {GPE_DEN_2D_XZ, "2d_xz.bin"}, {GPE_DEN_2D_YZ, "2d_yz.bin"},
                         {GPE_DEN_3D_XY0, "3d_xy0.bin"}, {GPE_DEN_3D_X0Z, "3d_x0z.bin"}, {GPE_DEN_3D_0YZ, "3d_0yz.bin"}};
   for (const Item &it : items) {
      check(gpe_density(s, it.kind, p.outstpx, p.outstpy, p.outstpz, buf.data(), (long) buf.size(), &cnt), "density");
      // imag3d names the NPAS z profile "...1d_z.txt" (imag:431)
      std::string suffix = (z_as_txt && it.kind == GPE_DEN_1D_Z) ? "1d_z.txt" : it.suffix;
      write_file(pre + suffix, buf.data(), (size_t) cnt);
   }
}

struct Obs {
   double norm = 0, mu = 0, en = 0, rms[4] = {0, 0, 0, 0}, c2 = 0;
};

void observe(gpe_solver *s, double g, double gd, Obs &o) {
   check(gpe_calcmuen(s, g, gd, &o.mu, &o.en), "calcmuen");
   check(gpe_calcrms(s, o.rms), "calcrms");
   check(gpe_psi_center2(s, &o.c2), "psi");
}

}  // namespace

int run_program(int mode, int argc, char **argv) {
   const auto t_start = std::chrono::steady_clock::now();
   double iter_time = 0.;
   const bool real = mode == 1;
   if (argc != 3 || std::strcmp(argv[1], "-i") != 0) {
      std::fprintf(stderr, "Usage: %s -i <input parameter file> \n", argv[0]);
      return EXIT_FAILURE;
   }
   if (!cfg_init(argv[2])) {
      std::fprintf(stderr, "Wrong input parameter file.\n");
      return EXIT_FAILURE;
   }
   Par p;
   readpar(mode, p);
   const double par = (p.opt == 2) ? 2. : 1.;

   gpe_params gp{};
   gp.mode = real ? GPE_MODE_REAL : GPE_MODE_IMAG;
   gp.precision = GPE_PREC_FP64;
   if (const char *pr = cfg_read("PRECISION")) gp.precision = (std::strcmp(pr, "MIXED") == 0) ? GPE_PREC_MIXED : GPE_PREC_FP64;
   gp.opt = p.opt;
   gp.device = p.device;
   gp.nx = p.Nx; gp.ny = p.Ny; gp.nz = p.Nz;
   gp.dx = p.dx; gp.dy = p.dy; gp.dz = p.dz; gp.dt = p.dt;
   gp.gamma = p.vgamma; gp.nu = p.vnu; gp.lambda = p.vlambda;
   gp.cutoff = p.cutoff;
   gpe_solver *s = nullptr;
   check(gpe_create(&gp, nullptr, &s), "solver creation");

   FILE *out = stdout;
   std::string fn;
   if (p.output) {
      fn = std::string(p.output) + ".txt";
      out = std::fopen(fn.c_str(), "w");
      if (!out) die("cannot open the output file\n");
   }
   FILE *frms = nullptr;
   if (p.rmsout) {
      fn = std::string(p.rmsout) + ".txt";
      frms = std::fopen(fn.c_str(), "w");
      if (!frms) die("cannot open the rms file\n");
   }
   FILE *dyna = nullptr;
   if (p.dynaout) {
      fn = std::string(p.dynaout) + ".txt";
      dyna = std::fopen(fn.c_str(), "w");
      if (!dyna) die("cannot open the dyna file\n");
   }

   std::fprintf(out, real ? " Real time propagation 3D,   OPTION = %d, MPI_NUM_PROCS = %d\n\n"
                          : " Imaginary time propagation 3D,   OPTION = %d, MPI_NUM_PROCS = %d\n\n", p.opt, 1);
   std::fprintf(out, "  Number of Atoms N = %li, Unit of length AHO = %.8f m\n", p.Na, p.aho);
   std::fprintf(out, "  Scattering length a = %.2f*a0, Dipolar ADD = %.2f*a0\n", p.as, p.add);
   std::fprintf(out, "  Nonlinearity G_3D = %.4f, Strength of DDI GD_3D = %.5f\n", p.g0, p.gd0);
   std::fprintf(out, "  Parameters of trap: GAMMA = %.2f, NU = %.2f, LAMBDA = %.2f\n\n", p.vgamma, p.vnu, p.vlambda);
   std::fprintf(out, " # Space Stp: NX = %li, NY = %li, NZ = %li\n", p.Nx, p.Ny, p.Nz);
   std::fprintf(out, "  Space Step: DX = %.6f, DY = %.6f, DZ = %.6f\n", p.dx, p.dy, p.dz);
   std::fprintf(out, " # Time Stp : NSTP = %li, NPAS = %li, NRUN = %li\n", p.Nstp, p.Npas, p.Nrun);
   std::fprintf(out, "   Time Step:   DT = %.6f\n", p.dt);
   std::fprintf(out, "   Dipolar Cut off:   R = %.3f\n\n", p.cutoff);
   if (real) std::fprintf(out, " * Change for dynamics: GPAR = %.3f, GDPAR = %.3f *\n\n", p.gpar, p.gdpar);
   std::fprintf(out, "                  --------------------------------------------------------\n");
   std::fprintf(out, "                    Norm      Chem        Ener/N     <r>     |Psi(0,0,0)|^2\n");
   std::fprintf(out, "                  --------------------------------------------------------\n");
   std::fflush(out);

   // couplings: imag3d leaves g = gd = 0 until the NSTP phase
   // (imag:309-317, 391-392); real3d sets them before initpsi (real:229-235).
   double g = 0., gd = 0.;
   if (real && p.Nstp == 0) { g = par * p.g0; gd = par * p.gd0; }

   if (real && p.Nstp == 0) {
      // initpsi reads imag3d-den.bin from the working directory (real:925-947)
      FILE *f = std::fopen("imag3d-den.bin", "rb");
      if (!f) {
         std::printf("Run the program using the input file to read. e.g.: imag3d-den.bin\n");
         return EXIT_FAILURE;
      }
      std::vector<double> rho((size_t) (p.Nx * p.Ny * p.Nz));
      const size_t got = std::fread(rho.data(), sizeof(double), rho.size(), f);
      std::fclose(f);
      if (got != rho.size()) {
         std::fprintf(stderr, "imag3d-den.bin holds %zu doubles, NX*NY*NZ = %zu are needed.\n", got, rho.size());
         return EXIT_FAILURE;
      }
      check(gpe_init_density(s, rho.data()), "initpsi");
   } else {
      check(gpe_init_gaussian(s), "initpsi");
   }

   Obs o;
   check(gpe_calcnorm(s, real ? 0 : 1, &o.norm), "calcnorm");
   observe(s, g, gd, o);
   std::fprintf(out, "Initial : %15.4f %11.5f %11.5f %10.5f %10.5f\n", o.norm, o.mu / par, o.en / par, o.rms[0], o.c2);
   std::fflush(out);
   auto rms_row = [&](const char *label, const Obs &ob) {
      if (frms) {
         std::fprintf(frms, "%s%12.5f %12.5f %12.5f %12.5f\n", label, ob.rms[0], ob.rms[1], ob.rms[2], ob.rms[3]);
         std::fflush(frms);
      }
   };
   auto rms_header = [&]() {
      if (!frms) return;
      std::fprintf(frms, real ? " Real time propagation 3D,   OPTION = %d\n\n" : " Imaginary time propagation 3D,   OPTION = %d\n\n",
                   p.opt);
      std::fprintf(frms, "                  --------------------------------------------------------\n");
      std::fprintf(frms, "Values of rms size:     <r>          <x>          <y>          <z>\n");
      std::fprintf(frms, "                  --------------------------------------------------------\n");
   };
   if (real) { rms_header(); rms_row("           Initial:", o); }
   if (p.initout) write_densities(s, p, p.initout, false);
   if (!real) { rms_header(); rms_row("           Initial:", o); }

   auto timed_run = [&](long n, double g_inc, double gd_inc, double *norm, long every, double *rbuf) {
      const auto t0 = std::chrono::steady_clock::now();
      check(gpe_run(s, n, &g, &gd, g_inc, gd_inc, norm, every, rbuf), "step loop");
      iter_time += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
   };
   auto phase_row = [&](const char *label, double norm) {
      observe(s, g, gd, o);
      if (real) check(gpe_calcnorm(s, 0, &norm), "calcnorm");
      std::fprintf(out, "%s%8.4f %11.5f %11.5f %10.5f %10.5f\n", label, norm, o.mu / par, o.en / par, o.rms[0], o.c2);
      std::fflush(out);
   };
   auto dyna_rows = [&](long n, const std::vector<double> &rb, double t0) {
      if (!dyna) return;
      for (long c = 0, q = 0; c < n; c += p.outstpt, q++)
         std::fprintf(dyna, "%8le   %8le   %8le   %8le   %8le\n", (c * p.dt + t0) * par, rb[4 * q], rb[4 * q + 1],
                      rb[4 * q + 2], rb[4 * q + 3]);
      std::fflush(dyna);
   };

   double norm = o.norm;
   // ---------------------------------------------------------------- NSTP
   if (p.Nstp != 0) {
      double g_stp = par * p.g0 / (double) p.Nstp, gd_stp = par * p.gd0 / (double) p.Nstp;
      g = 0.; gd = 0.;
      timed_run(p.Nstp, g_stp, gd_stp, &norm, 0, nullptr);
      phase_row("After NSTP iter.:", norm);
      rms_row("  After NSTP iter.:", o);
      if (p.nstpout) write_densities(s, p, p.nstpout, false);
   } else {
      g = par * p.g0;
      gd = par * p.gd0;
   }
   // ---------------------------------------------------------------- NPAS
   {
      const bool dy = dyna && p.outstpt > 0;
      std::vector<double> rb(dy ? (size_t) (4 * ((p.Npas + p.outstpt - 1) / p.outstpt) + 4) : 0);
      timed_run(p.Npas, 0., 0., &norm, dy ? p.outstpt : 0, dy ? rb.data() : nullptr);
      if (dy) dyna_rows(p.Npas, rb, 0.);
      phase_row("After NPAS iter.:", norm);
      if (real) rms_row("  After NPAS iter.:", o);
      if (p.npasout) write_densities(s, p, p.npasout, !real);
      if (!real) rms_row("  After NPAS iter.:", o);
   }
   // quench (real:493-494)
   if (real) { g = p.gpar * g; gd = p.gdpar * gd; }
   // ---------------------------------------------------------------- NRUN
   {
      const bool dy = dyna && p.outstpt > 0;
      std::vector<double> rb(dy ? (size_t) (4 * ((p.Nrun + p.outstpt - 1) / p.outstpt) + 4) : 0);
      timed_run(p.Nrun, 0., 0., &norm, dy ? p.outstpt : 0, dy ? rb.data() : nullptr);
      if (dy) dyna_rows(p.Nrun, rb, p.dt * p.Npas);
      phase_row("After NRUN iter.:", norm);
      if (real) {
         rms_row("  After NRUN iter.:", o);
         if (frms) std::fprintf(frms, "                  --------------------------------------------------------\n");
         if (p.nrunout) write_densities(s, p, p.nrunout, false);
      } else {
         if (p.nrunout) write_densities(s, p, p.nrunout, false);
         rms_row("  After NRUN iter.:", o);
         if (frms) std::fprintf(frms, "                  --------------------------------------------------------\n");
      }
   }
   if (frms) std::fclose(frms);
   if (dyna) std::fclose(dyna);
   std::fprintf(out, "                  --------------------------------------------------------\n\n");
   gpe_destroy(s);
   const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
   std::fprintf(out, " Initialization/allocation wall-clock time: %.3f seconds\n", wall - iter_time);
   std::fprintf(out, " Calculation (iterations) wall-clock time: %.3f seconds\n", iter_time);
   if (p.output) std::fclose(out);
   return EXIT_SUCCESS;
}

}  // namespace gpecli
