// castro_main.cu -- the mini-app driver (Source/main.cpp) on the B200 library.
//
// Same command-line keys as the reference (key=value, ParmParse style):
//   n_cell, max_box_size (64), min_box_size (16), max_level (0, only 0 is
//   supported), stop_time (0.01), max_step (10000000), fom (1),
//   diagnostic_interval (50)
// plus keys for what the reference hard-codes:
//   problem=reference|sedov   (Source/Prob.F90 constants, or the unit-cube
//                              configuration: rho, T, E, r = 4 zones, X = 0.5/0.5)
//   nspec=13|2, bc=periodic|outflow, mode=batched|persistent|plain|plain_box,
//   table=<helm_table.dat>
//   rho, T, E (sedov problem constants)
//   momentum_flux_pressure=0|1 (1: the interface pressure in the normal
//                              momentum flux, as full Castro has it; the
//                              reference, and the default, have none)
//   use_eos_coulomb=0|1        (1: Coulomb corrections in the EOS, as the
//                              reference's 2017 runs had them; its eos.F90,
//                              and the default, have none)
// and prints the reference's progress lines and figure of merit.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <chrono>
#include <map>
#include <string>
#include <vector>

#include "../../include/castro_b200.h"

namespace {

std::vector<int> chop(int n, int max_size)
{
    int k = (n + max_size - 1) / max_size;
    if (k < 1) k = 1;
    std::vector<int> out;
    int base = n / k, rem = n % k;
    for (int i = 0; i < k; ++i) out.push_back(base + (i < rem ? 1 : 0));
    return out;
}

void usage()
{
    printf("\nmini-Castro is an astrophysical 3D Sedov-Taylor blast wave benchmark.\n");
    printf("The algorithm closely resembles that of the Castro code.\n\n");
    printf("This mini-app has several inputs parameters (values in parentheses are the defaults):\n\n");
    printf("n_cell: The number of zones per dimension. This parameter must be set to run the code.\n");
    printf("max_box_size (64): The maximum size of a box in the domain.\n");
    printf("min_box_size (16): The minimum size of a box in the domain.\n");
    printf("max_level (0): The maximum adaptive mesh refinement level (zero-indexed).\n");
    printf("stop_time (0.01): The stopping time of the simulation, in seconds.\n");
    printf("max_step (10000000): The maximum number of timesteps to take.\n\n");
    printf("B200 additions: problem=reference|sedov nspec=13|2 bc=periodic|outflow\n"
           "               mode=batched|persistent|plain|plain_box table=<path>\n"
           "               plot_file=<dir> (AMReX plotfile of the final state)\n"
           "               momentum_flux_pressure=0|1 (1: pressure in the momentum flux, as full Castro)\n"
           "               use_eos_coulomb=0|1 (1: Coulomb corrections in the EOS)\n\n");
}

}  // namespace

extern "C" int castro_main(int argc, char** argv)
{
    std::map<std::string, std::string> kv;
    for (int a = 1; a < argc; ++a) {
        const char* eq = strchr(argv[a], '=');
        if (!eq) continue;
        kv[std::string(argv[a], eq - argv[a])] = std::string(eq + 1);
    }
    auto geti = [&](const char* k, long long d) { return kv.count(k) ? atoll(kv[k].c_str()) : d; };
    auto getd = [&](const char* k, double d) { return kv.count(k) ? atof(kv[k].c_str()) : d; };
    auto gets = [&](const char* k, const char* d) { return kv.count(k) ? kv[k] : std::string(d); };

    int n_cell = (int)geti("n_cell", 0);
    if (n_cell <= 0) { usage(); return 0; }
    printf("\nStarting mini-Castro...\n\n");
    long long max_step = geti("max_step", 10000000);
    double stop_time = getd("stop_time", 1.0e-2);
    int do_fom = (int)geti("fom", 1);
    int max_box = (int)geti("max_box_size", 64);
    int min_box = (int)geti("min_box_size", 16);
    int max_level = (int)geti("max_level", 0);
    int diag = (int)geti("diagnostic_interval", 50);
    std::string problem = gets("problem", "reference");
    int nspec = (int)geti("nspec", problem == "reference" ? 13 : 2);
    int bc = gets("bc", problem == "reference" ? "periodic" : "outflow") == "periodic" ? CASTRO_BC_PERIODIC : CASTRO_BC_OUTFLOW;
    const std::string mode_s = gets("mode", "batched");
    int mode = CASTRO_MODE_BATCHED;
    if (mode_s == "plain") mode = CASTRO_MODE_PLAIN;
    else if (mode_s == "plain_box") mode = CASTRO_MODE_PLAIN_BOX;
    else if (mode_s == "persistent") mode = CASTRO_MODE_PERSISTENT;
    else if (mode_s != "batched") {
        fprintf(stderr, "mode must be batched, persistent, plain or plain_box\n");
        return 1;
    }
    if (max_level != 0) { fprintf(stderr, "max_level > 0 is not supported (single-level advance only)\n"); return 1; }

    printf("Initializing AMR driver using the following runtime parameters:\n\n");
    printf("n_cell = %d\nmax_box_size = %d\nmin_box_size = %d\nmax_level = %d\nmax_step = %lld\nstop_time = %g\n\n",
           n_cell, max_box, min_box, max_level, max_step, stop_time);

    if (nspec == 13) network_init();
    else {
        const double a[2] = {4.0, 16.0}, z[2] = {2.0, 8.0};
        castro_network_init(2, a, z);
    }
    castro_set_momentum_flux_pressure((int)geti("momentum_flux_pressure", 0));
    castro_set_coulomb_corrections((int)geti("use_eos_coulomb", 0));
    std::string table = gets("table", getenv("CASTRO_HELM_TABLE") ? getenv("CASTRO_HELM_TABLE") : "helm_table.dat");
    if (castro_eos_init_path(table.c_str()) != CASTRO_OK) {
        fprintf(stderr, "eos_init: %s\n", castro_error_string());
        return 1;
    }

    castro_instance_desc D;
    memset(&D, 0, sizeof D);
    double L = problem == "reference" ? 1.0e9 : 1.0;   // Source/main.cpp:80-81
    for (int d = 0; d < 3; ++d) { D.dom_lo[d] = 0; D.dom_hi[d] = n_cell - 1; D.problo[d] = 0.0; D.probhi[d] = L; }
    D.bc = bc;
    std::vector<int> s = chop(n_cell, max_box);
    std::vector<int> blo, bhi;
    int z0 = 0;
    for (int nz : s) {
        int y0 = 0;
        for (int ny : s) {
            int x0 = 0;
            for (int nx : s) {
                blo.insert(blo.end(), {x0, y0, z0});
                bhi.insert(bhi.end(), {x0 + nx - 1, y0 + ny - 1, z0 + nz - 1});
                x0 += nx;
            }
            y0 += ny;
        }
        z0 += nz;
    }
    D.nbox = (int)(blo.size() / 3);
    D.box_lo = blo.data();
    D.box_hi = bhi.data();
    castro_problem_defaults(&D.prob);
    if (problem != "reference") {
        D.prob.ambient_from_T = 1;
        D.prob.dens_ambient = getd("rho", 1.0);
        D.prob.T_ambient = getd("T", 1.0e6);
        D.prob.exp_energy = getd("E", 1.0e50);
        D.prob.r_init = 4.0 * L / n_cell;
        D.prob.X[0] = 0.5;
        D.prob.X[1] = 0.5;
    }
    D.stop_time = stop_time;

    castro_sim* sim = castro_sim_create(1, &D, mode);
    if (!sim) { fprintf(stderr, "castro_sim_create: %s\n", castro_error_string()); return 1; }
    printf("Running simulation and calculating diagnostics every %d timesteps...\n\n", diag);
    castro_sim_init_data(sim);
    auto t1 = std::chrono::steady_clock::now();
    long long nsteps = 0;
    while ((nsteps < max_step || max_step < 0) && (castro_sim_time(sim, 0) < stop_time || stop_time < 0.0)) {
        if (castro_sim_step(sim) != CASTRO_OK) { fprintf(stderr, "step: %s\n", castro_error_string()); return 1; }
        ++nsteps;
        if (diag > 0 && nsteps % diag == 0) {
            double bm;
            double r = castro_sim_blast_radius(sim, 0, &bm);
            printf("Blast radius at step %lld, time %e: %.3f km\n", nsteps, castro_sim_time(sim, 0), r / 1.0e5);
        }
    }
    castro_sim_sync(sim);
    const std::string plot = gets("plot_file", "");
    if (!plot.empty() && castro_sim_write_plotfile(sim, 0, plot.c_str()) != CASTRO_OK)
        fprintf(stderr, "plotfile: %s\n", castro_error_string());
    double zones = (double)n_cell * n_cell * n_cell;
    castro_sim_destroy(sim);
    auto t2 = std::chrono::steady_clock::now();
    double runtime = std::chrono::duration<double>(t2 - t1).count();
    double fom = zones * (double)nsteps / runtime / 1.e6;
    printf("\nSimulation completed!\nNumber of timesteps taken: %lld\n\n", nsteps);
    if (do_fom) printf("Figure of Merit (zones / usec): %.3f\n\n", fom);
    return 0;
}
