// adapter_run -- the reference's own LFIntegrator driving the GPU force
// objects of swinmd_b200/adapter/swinmd_gpu.h, for the drop-in test
// (tests/test_gpu_adapter.py).  Test infrastructure: built by
// oracle/Makefile against the reference's sources, run on a GPU box.
//
// Usage, inside a case directory (config.txt, sysData.in, coordinates):
//     adapter_run <nsteps> <out> [mixed]
// writes the same records as `ref_dump run` (name count values per line):
// per-step potential energy, kinetic energy, temperature, zeta, list
// updates and atomic pressure tensor, then the final positions and
// velocities.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>
#include "mpi.h"
#include "swinmd_gpu.h"

int mpi_size_g = 1;
int mpi_rank_g = 0;

static FILE *g_out = nullptr;

static void rec(const char *name, const std::vector<double> &v) {
    fprintf(g_out, "%s %zu", name, v.size());
    for (double x : v) fprintf(g_out, " %.17g", x);
    fputc('\n', g_out);
}

int main(int argc, char **argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: adapter_run <nsteps> <out> [mixed]\n");
        return 2;
    }
    const int nsteps = atoi(argv[1]);
    const int precision = argc > 3 && !strcmp(argv[3], "mixed") ? SMD_PREC_MIXED : SMD_PREC_FP64;
    // the set-up of Simulation::setup_simulation (src/Simulation.cpp:171-263)
    // without its output files
    SimConfiguration *cfg = new SimConfiguration((char *)"config.txt");
    cfg->read_config_file();
    Parameters *params = new Parameters(cfg->get_sysData_file());
    Ensemble *ens = new Ensemble();
    ens->set_mol_system(params);
    ens->set_configuration(cfg);
    ens->compute_bound_box();
    ens->set_pairlist();
    ens->set_sysdata_file(new std::ofstream("sysData.out", std::ios::out));
    ens->set_result_file(new std::ofstream("result.out", std::ios::out));

    swinmd_gpu::GpuPath path(ens, precision);
    swinmd_gpu::GpuForceLFIntegrator *lf = new swinmd_gpu::GpuForceLFIntegrator(ens, cfg, &path);
    g_out = fopen(argv[2], "w");
    std::vector<double> epot, ekin, atemp, zeta, nupd, ptensor, molpt;
    for (int k = 0; k < nsteps; k++) {
        lf->run(1);
        const Energy &E = ens->myEnergy;
        epot.push_back(E.totEnergy);
        ekin.push_back(E.atomKinEnergy);
        atemp.push_back(ens->atomTemp);
        zeta.push_back(lf->zeta());
        nupd.push_back(lf->list_updates());
        for (int q = 0; q < 9; q++) ptensor.push_back(ens->atomPressure[q]);
        molpt.push_back(lf->lustig_pressure());
    }
    rec("step_epot", epot);
    rec("step_ekin", ekin);
    rec("step_atomtemp", atemp);
    rec("step_zeta", zeta);
    rec("step_nupdates", nupd);
    rec("step_atompressure", ptensor);
    rec("step_molpt", molpt);
    const int n = ens->nAtoms;
    std::vector<double> p(3 * n), v(3 * n);
    for (int i = 0; i < n; i++) {
        p[3 * i] = ens->atoms[i].position.x;
        p[3 * i + 1] = ens->atoms[i].position.y;
        p[3 * i + 2] = ens->atoms[i].position.z;
        v[3 * i] = ens->atoms[i].velocity.x;
        v[3 * i + 1] = ens->atoms[i].velocity.y;
        v[3 * i + 2] = ens->atoms[i].velocity.z;
    }
    rec("final_pos", p);
    rec("final_vel", v);
    fclose(g_out);
    return 0;
}
