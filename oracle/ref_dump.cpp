// ref_dump — drives the reference SwinMD objects (built by oracle/Makefile)
// and writes their FP64 results as text records, one per line:
//     <name> <count> v0 v1 ... v(count-1)
// Test infrastructure only: the checker that pins this project's CPU
// restatement and its CUDA path.  It never runs inside the product.
//
// Usage (run inside a case directory holding config.txt, sysData.in and the
// coordinate file the config names):
//     ref_dump forces <out>        one force evaluation of every term the
//                                  config enables, each term on its own
//     ref_dump run <nsteps> <out>  LFIntegrator::start() then nsteps x run(1)
//     ref_dump mie <out>           MieForce::compute() on its own
//     ref_dump buck <out>          BuckinghamForce::compute() on its own
//     ref_dump saap <out>          SAAPForce::compute() on its own (three atom types)
//     ref_dump rdf <out>           one RDF::sampling() of the configuration
//     ref_dump nhrun <nsteps> <out> NHIntegrator::start() then nsteps x run(1)
//
// Setup follows Simulation::setup_simulation (src/Simulation.cpp:171-263)
// without the output files.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <ctime>
#include <cstdint>
#include <iostream>
#include <iomanip>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include <set>
#include <map>
#include <algorithm>
#include <utility>
#include <limits>
#include "mpi.h"
// Several members the checker reads (LFIntegrator::vtMinus, the force
// objects' virial) are private; widen access for this translation unit only.
#define class struct
#define private public
#define protected public
#include "Ensemble.h"
#include "Parameters.h"
#include "SimConfiguration.h"
#include "Integrator.h"
#include "integrators/LFIntegrator.h"
#include "integrators/NHIntegrator.h"
#include "forces/LJForce.h"
#include "forces/MieForce.h"
#include "forces/BuckinghamForce.h"
#include "forces/SAAPForce.h"
#include "forces/BuffvdWForce.h"
#include "forces/EwaldForce.h"
#include "forces/WolfForce.h"
#include "forces/Multipole.h"
#include "forces/Induction.h"
#include "forces/BondForce.h"
#include "forces/AngleForce.h"
#include "forces/UreyBradleyForce.h"
#include "observables/RDF.h"
#undef class
#undef private
#undef protected

int mpi_size_g = 1;
int mpi_rank_g = 0;

static FILE *g_out = nullptr;

static void rec(const char *name, const std::vector<double> &v) {
    fprintf(g_out, "%s %zu", name, v.size());
    for (double x : v) fprintf(g_out, " %.17g", x);
    fputc('\n', g_out);
}
static void rec1(const char *name, double x) { rec(name, std::vector<double>{x}); }

struct Setup {
    SimConfiguration *cfg;
    Parameters *params;
    Ensemble *ens;
};

static Setup build() {
    Setup s;
    s.cfg = new SimConfiguration((char *)"config.txt");
    s.cfg->read_config_file();
    s.params = new Parameters(s.cfg->get_sysData_file());
    s.ens = new Ensemble();
    s.ens->set_mol_system(s.params);
    s.ens->set_configuration(s.cfg);
    s.ens->compute_bound_box();
    s.ens->set_pairlist();
    s.ens->set_sysdata_file(new std::ofstream("sysData.out", std::ios::out));
    s.ens->set_result_file(new std::ofstream("result.out", std::ios::out));
    return s;
}

static void dump_state(Ensemble *e, const char *tag) {
    int n = e->nAtoms;
    std::vector<double> p(3 * n), v(3 * n);
    for (int i = 0; i < n; i++) {
        p[3 * i] = e->atoms[i].position.x;
        p[3 * i + 1] = e->atoms[i].position.y;
        p[3 * i + 2] = e->atoms[i].position.z;
        v[3 * i] = e->atoms[i].velocity.x;
        v[3 * i + 1] = e->atoms[i].velocity.y;
        v[3 * i + 2] = e->atoms[i].velocity.z;
    }
    std::string a = std::string(tag) + "_pos", b = std::string(tag) + "_vel";
    rec(a.c_str(), p);
    rec(b.c_str(), v);
}

static void dump_pairs(Ensemble *e) {
    std::vector<double> pr;
    for (int i = 0; i < e->nAtoms; i++) {
        Atom *a = &e->atoms[i];
        for (int k = 0; k < a->get_list_size(); k++) {
            int j = a->myPairList[k]->atomID;
            pr.push_back(std::min(i, j));
            pr.push_back(std::max(i, j));
        }
    }
    rec("pairs", pr);
}

static void zero(Ensemble *e) {
    for (int i = 0; i < e->nAtoms; i++) e->atoms[i].force = 0.0;
    for (int k = 0; k < 9; k++) {
        e->virial[k] = 0.0;
        e->longVirial[k] = 0.0;
    }
    std::memset(&e->myEnergy, 0, sizeof(e->myEnergy));
}

static void dump_forces(Ensemble *e, const char *tag) {
    int n = e->nAtoms;
    std::vector<double> f(3 * n);
    for (int i = 0; i < n; i++) {
        f[3 * i] = e->atoms[i].force.x;
        f[3 * i + 1] = e->atoms[i].force.y;
        f[3 * i + 2] = e->atoms[i].force.z;
    }
    std::string a = std::string(tag) + "_force";
    rec(a.c_str(), f);
    std::string b = std::string(tag) + "_virial";
    rec(b.c_str(), std::vector<double>(e->virial, e->virial + 9));
    std::string c = std::string(tag) + "_longvirial";
    rec(c.c_str(), std::vector<double>(e->longVirial, e->longVirial + 9));
    const Energy &E = e->myEnergy;
    std::string d = std::string(tag) + "_energy";
    // order: lj real long correct molCorrect surfCorrect realPol longPol
    //        correctPol molCorrectPol surfacePol bond angle ub
    rec(d.c_str(), {E.ljEnergy, E.realEnergy, E.longEnergy, E.correctEnergy,
                    E.molCorrectEnergy, E.surfCorrectEnergy, E.realPolEnergy,
                    E.longPolEnergy, E.correctPolEnergy, E.molCorrectPolEnergy,
                    E.surfacePolEnergy, E.bondEnergy, E.angleEnergy, E.ubEnergy});
}

static void header(Setup &s) {
    Ensemble *e = s.ens;
    rec("box", {e->boxLx, e->boxLy, e->boxLz});
    rec1("natoms", e->nAtoms);
    rec1("pair_cutoff2", e->pairCutOff);
    std::vector<double> m(e->nAtoms), q(e->nAtoms), t(e->nAtoms), mol(e->nAtoms);
    for (int i = 0; i < e->nAtoms; i++) {
        m[i] = e->atoms[i].mass;
        q[i] = e->atoms[i].scaledCharge;
        t[i] = e->atoms[i].atomType;
        mol[i] = e->atoms[i].molID;
    }
    rec("mass", m);
    rec("scaled_charge", q);
    rec("type", t);
    rec("molid", mol);
    dump_state(e, "init");
    dump_pairs(e);
}

static int mode_forces(const char *out) {
    Setup s = build();
    g_out = fopen(out, "w");
    header(s);
    Ensemble *e = s.ens;
    SimConfiguration *c = s.cfg;
    if (c->compute_buffamoeba()) {
        zero(e);
        BuffvdWForce f(e);
        f.compute();
        dump_forces(e, "buff");
    } else {
        zero(e);
        LJForce f(e);
        f.compute();
        dump_forces(e, "lj");
        if (c->compute_lustig()) {
            const Lustig &L = e->myLustig;
            rec("lustig_lj", std::vector<double>{L.ljUlus, L.ljdUlus, L.ljd2Ulus});
        }
    }
    if (c->compute_wolf()) {
        zero(e);
        WolfForce f(e);
        f.compute();
        dump_forces(e, "wolf");
    }
    if (c->compute_ewald_force()) {
        zero(e);
        EwaldForce f(e);
        f.compute();
        dump_forces(e, "ewald_short");
        zero(e);
        f.compute_long();
        dump_forces(e, "ewald_long");
        rec1("ewald_nk", (double)f.kVector.size());
    }
    if (c->compute_multipol()) {
        zero(e);
        Multipole mp(e);
        mp.compute();
        dump_forces(e, "mp_short");
        {
            int n = e->nAtoms;
            std::vector<double> dip(3 * n), quad(6 * n);
            for (int i = 0; i < n; i++) {
                dip[3 * i] = mp.myL2G->dip[i].x;
                dip[3 * i + 1] = mp.myL2G->dip[i].y;
                dip[3 * i + 2] = mp.myL2G->dip[i].z;
                quad[6 * i] = mp.myL2G->Qxx[i];
                quad[6 * i + 1] = mp.myL2G->Qxy[i];
                quad[6 * i + 2] = mp.myL2G->Qxz[i];
                quad[6 * i + 3] = mp.myL2G->Qyy[i];
                quad[6 * i + 4] = mp.myL2G->Qyz[i];
                quad[6 * i + 5] = mp.myL2G->Qzz[i];
            }
            rec("mp_dip", dip);
            rec("mp_quad", quad);
            rec("mp_parts", {mp.selfEnergy, mp.realEnergy, mp.intraMolEnergy});
        }
        zero(e);
        mp.compute_long();
        dump_forces(e, "mp_long");
        if (c->compute_induction()) {
            zero(e);
            Induction ind(e);
            ind.compute();
            dump_forces(e, "ind_short");
            int n3 = 3 * e->nAtoms;
            rec("ind_E0", std::vector<double>(ind.Ei0, ind.Ei0 + n3));
            rec("ind_P", std::vector<double>(ind.Pi, ind.Pi + n3));
            rec("ind_parts", {ind.selfEnergy, ind.realEnergy, ind.intraMolEnergy});
            zero(e);
            ind.compute_long();
            dump_forces(e, "ind_long");
        }
    }
    // bonded terms of flexible molecules (Integrator::initialise,
    // src/Integrator.cpp:163-190)
    if (!c->is_constraint_on() && e->nBonds > 0) {
        zero(e);
        BondForce f(e);
        f.compute();
        dump_forces(e, "bond");
    }
    if (!c->is_constraint_on() && e->nAngles > 0) {
        zero(e);
        AngleForce f(e);
        f.compute();
        dump_forces(e, "angle");
    }
    if (c->compute_harmonic_ub()) {
        zero(e);
        UreyBradleyForce f(e);
        f.compute();
        dump_forces(e, "ub");
    }
    fclose(g_out);
    return 0;
}

static int mode_single(const char *which, const char *out) {
    Setup s = build();
    g_out = fopen(out, "w");
    header(s);
    Ensemble *e = s.ens;
    zero(e);
    if (!strcmp(which, "mie")) {
        MieForce f(e);
        f.compute();
        dump_forces(e, "mie");
    } else if (!strcmp(which, "saap")) {
        // SAAPForce with its built-in three-type table (SAAPForce.h); the
        // table is recorded so that the GPU side runs the same parameters
        SAAPForce f(e);
        f.compute();
        dump_forces(e, "saap");
        std::vector<double> tab;
// (WolfForce.h defines a macro of the first field's name)
#pragma push_macro("Aa0")
#undef Aa0
        for (int k = 0; k < e->nAtomTypes * e->nAtomTypes; k++) {
            const SAAPParam &q = f.saapParams[k];
            for (double v : {q.Aa0, q.Aa1, q.Aa2, q.Aa3, q.Aa4, q.Aa5}) tab.push_back(v);
        }
#pragma pop_macro("Aa0")
        rec("saap_params", tab);
    } else {
        BuckinghamForce f(e);
        f.compute();
        dump_forces(e, "buck");
    }
    fclose(g_out);
    return 0;
}

static int mode_run(int nsteps, const char *out) {
    Setup s = build();
    g_out = fopen(out, "w");
    header(s);
    Ensemble *e = s.ens;
    LFIntegrator *lf = new LFIntegrator(e, s.cfg);  // runs start(): F(0), vtMinus
    dump_forces(e, "start");
    {
        std::vector<double> vm(3 * e->nAtoms);
        for (int i = 0; i < e->nAtoms; i++) {
            vm[3 * i] = lf->vtMinus[i].x;
            vm[3 * i + 1] = lf->vtMinus[i].y;
            vm[3 * i + 2] = lf->vtMinus[i].z;
        }
        rec("start_vtminus", vm);
    }
    std::vector<double> epot, ekin, atemp, zeta, press, nupd;
    std::vector<double> ptensor, mtensor, lus, lus_all, molvirt, molpt;
    double run_seconds = 0.0;
    for (int k = 0; k < nsteps; k++) {
        timespec t0, t1;
        clock_gettime(CLOCK_MONOTONIC, &t0);
        lf->run(1);
        clock_gettime(CLOCK_MONOTONIC, &t1);
        run_seconds += (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
        if (s.cfg->compute_lustig()) {
            // the LJ term's Lustig values of this step's forces (evaluated
            // at the positions the previous step left, with its centres)
            const Lustig &L = e->myLustig;
            for (double v : {L.ljUlus, L.ljdUlus, L.ljd2Ulus}) lus.push_back(v);
            // every field of Ensemble::myLustig in declaration order (each
            // force term writes its own fields during the step)
            const double *all = reinterpret_cast<const double *>(&L);
            static_assert(sizeof(Lustig) == 29 * sizeof(double), "Lustig layout");
            lus_all.insert(lus_all.end(), all, all + 29);
            if (k == 0) dump_state(e, "step_after1");
        }
        // the step's Lustig virial and pressure (LFIntegrator.cpp:731-741)
        molvirt.push_back(lf->molVirt);
        molpt.push_back(lf->molPt);
        const Energy &E = e->myEnergy;
        epot.push_back(E.totEnergy);
        ekin.push_back(E.atomKinEnergy);
        atemp.push_back(e->atomTemp);
        zeta.push_back(lf->fnh);
        nupd.push_back(lf->numUpdates);
        for (int q = 0; q < 9; q++) ptensor.push_back(e->atomPressure[q]);
        for (int q = 0; q < 9; q++) mtensor.push_back(e->molPressure[q]);
    }
    if (!lus.empty()) rec("step_lustig", lus);
    if (!lus_all.empty()) rec("step_lustig_all", lus_all);
    rec("step_molvirt", molvirt);
    rec("step_molpt", molpt);
    rec("step_epot", epot);
    rec("step_ekin", ekin);
    rec("step_atomtemp", atemp);
    rec("step_zeta", zeta);
    rec("step_nupdates", nupd);
    rec("step_atompressure", ptensor);
    rec("step_molpressure", mtensor);
    rec1("run_seconds", run_seconds);
    dump_state(e, "final");
    dump_forces(e, "final");
    {
        std::vector<double> vm(3 * e->nAtoms);
        for (int i = 0; i < e->nAtoms; i++) {
            vm[3 * i] = lf->vtMinus[i].x;
            vm[3 * i + 1] = lf->vtMinus[i].y;
            vm[3 * i + 2] = lf->vtMinus[i].z;
        }
        rec("final_vtminus", vm);
    }
    fclose(g_out);
    return 0;
}

// NHIntegrator (the chain, with the barostat when the config asks for
// ensemble 1): its start, then nsteps x run(1), with the chain and barostat
// variables after every step
static int mode_nhrun(int nsteps, const char *out) {
    Setup s = build();
    g_out = fopen(out, "w");
    header(s);
    Ensemble *e = s.ens;
    NHIntegrator *nh = new NHIntegrator(e, s.cfg);  // runs start(): F(0)
    std::vector<double> epot, ekin, atemp, vol, boxl, vlog, vnh, molvirt, molpt, ptensor;
    for (int k = 0; k < nsteps; k++) {
        nh->run(1);
        const Energy &E = e->myEnergy;
        epot.push_back(E.totEnergy);
        ekin.push_back(E.atomKinEnergy);
        atemp.push_back(e->atomTemp);
        boxl.push_back(e->boxLx);
        vol.push_back(e->boxLx * e->boxLy * e->boxLz);
        vlog.push_back(nh->vlog);
        for (int q = 0; q < 4; q++) vnh.push_back(nh->vnh[q]);
        molvirt.push_back(nh->molVirt);
        molpt.push_back(nh->molPt);
        for (int q = 0; q < 9; q++) ptensor.push_back(e->atomPressure[q]);
    }
    rec("nh_epot", epot);
    rec("nh_ekin", ekin);
    rec("nh_atomtemp", atemp);
    rec("nh_boxl", boxl);
    rec("nh_volume", vol);
    rec("nh_vlog", vlog);
    rec("nh_vnh", vnh);
    rec("nh_molvirt", molvirt);
    rec("nh_molpt", molpt);
    rec("nh_atompressure", ptensor);
    dump_state(e, "nh_final");
    fclose(g_out);
    return 0;
}

// one RDF::sampling of the current configuration: the raw histogram
// rdfTable[t1][t2][bin] (both orders of every pair), the bin count and the
// per-type counts (src/observables/RDF.cpp:109-144)
static int mode_rdf(const char *out) {
    Setup s = build();
    g_out = fopen(out, "w");
    header(s);
    Ensemble *e = s.ens;
    RDF rdf(e, 1 << 30);
    rdf.sampling();
    const int nt = e->nAtomTypes;
    std::vector<double> h;
    for (int a = 0; a < nt; a++)
        for (int b = 0; b < nt; b++)
            for (int k = 0; k < rdf.nBins; k++) h.push_back(rdf.rdfTable[a][b][k]);
    rec("rdf_hist", h);
    rec1("rdf_nbins", rdf.nBins);
    rec1("rdf_maxr", rdf.maxR);
    std::vector<double> npt(rdf.numPerType, rdf.numPerType + nt);
    rec("rdf_numpertype", npt);
    fclose(g_out);
    return 0;
}

int main(int argc, char **argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: ref_dump forces|mie|buck <out> | run <nsteps> <out>\n");
        return 2;
    }
    if (!strcmp(argv[1], "forces")) return mode_forces(argv[2]);
    if (!strcmp(argv[1], "mie") || !strcmp(argv[1], "buck") || !strcmp(argv[1], "saap"))
        return mode_single(argv[1], argv[2]);
    if (!strcmp(argv[1], "run") && argc >= 4) return mode_run(atoi(argv[2]), argv[3]);
    if (!strcmp(argv[1], "rdf")) return mode_rdf(argv[2]);
    if (!strcmp(argv[1], "nhrun") && argc >= 4) return mode_nhrun(atoi(argv[2]), argv[3]);
    fprintf(stderr, "unknown mode\n");
    return 2;
}
