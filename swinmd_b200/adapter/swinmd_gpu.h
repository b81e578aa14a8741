// swinmd_gpu.h -- the C++ adapter that puts SwinMD's force terms on the B200
// path, through the C ABI of libswinmd_b200.so (include/swinmd_b200.h).
//
// It sits beside the reference's own classes and changes none of them:
//
//   GpuPath                one smd_ctx per Ensemble, set up from the
//                          reference's Ensemble / Parameters /
//                          SimConfiguration objects (Simulation::setup_simulation,
//                          src/Simulation.cpp:171-263)
//   GpuLJForce             LJForce::compute (src/forces/LJForce.cpp:58-255)
//   GpuEwaldForce          EwaldForce::compute / compute_long
//                          (src/forces/EwaldForce.cpp:127-196)
//   GpuForceLFIntegrator   the reference's own LFIntegrator (leap-frog, Nose-Hoover,
//                          SHAKE on the host) driving the GPU force objects: the
//                          pointers Integrator::initialise filled
//                          (src/Integrator.cpp:111-203) are swapped for the
//                          GPU ones, and LFIntegrator::run calls them as
//                          before (src/integrators/LFIntegrator.cpp:387-458)
//
// Every GPU force object honours the output conventions of the class it
// replaces: forces add into Atom::force, energies are assigned into
// Ensemble::myEnergy, the short-range virial goes into Ensemble::virial with
// the reference's sign, and the reciprocal virial into Ensemble::longVirial
// (components 0..7, as EwaldForce::compute_long copies them).  Errors of the
// C ABI become the reference's ERRORMSG (src/Errors.h:53-62).
//
// Positions are uploaded when they differ from the last upload; the library
// keeps its pair list while every site stays within half the skin, as the
// reference's integrator does.
#ifndef SWINMD_GPU_H
#define SWINMD_GPU_H

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

// the C ABI first: a reference header defines a macro `polar`
#include "swinmd_b200.h"
#include "Ensemble.h"
#include "Errors.h"
#include "Parameters.h"
#include "SimConfiguration.h"
#include "integrators/LFIntegrator.h"
#include "forces/EwaldForce.h"
#include "forces/LJForce.h"

namespace swinmd_gpu {

inline void check(smd_ctx *ctx, int rc, const char *what) {
    if (rc != SMD_OK) {
        const std::string m = std::string(what) + ": " + (ctx ? smd_last_error(ctx) : "no context");
        ERRORMSG(m.c_str());
    }
}

// The dispersion tail of LJForce::long_range_correct
// (src/forces/LJForce.cpp:260-370): energy and virial corrections, from the
// same type counts, pair parameters and exclusions.
inline void lj_tail(Ensemble *e, double *e_lrc, double *v_lrc) {
    const int nt = e->nAtomTypes, n = e->nAtoms;
    std::vector<long long> count(nt, 0);
    for (int i = 0; i < n; i++) count[e->atoms[i].atomType]++;
    double csix = 0.0;
    long long npair = 0, nexcl = 0;
    for (int i = 0; i < nt; i++)
        for (int j = i; j < nt; j++) {
            const LJPairParam p = e->myParams->get_lj_parameter(i, j);
            const long long nij = i != j ? count[i] * count[j] : (long long)(count[i] * (count[i] - 1) * 0.5);
            csix += nij * p.eps * p.sigma * p.sigma * p.sigma;
            npair += nij;
        }
    for (int i = 0; i < n; i++)
        for (int k = 0; e->exclusionTable[i][k] != -1; k++) {
            const int j = e->exclusionTable[i][k];
            if (j < i) continue;
            const LJPairParam p = e->myParams->get_lj_parameter(e->atoms[i].atomType, e->atoms[j].atomType);
            csix -= p.eps * p.sigma * p.sigma * p.sigma;
            nexcl++;
        }
    csix = npair - nexcl <= 0 ? 0.0 : csix / (double)(npair - nexcl);
    const double rc = e->myConfig->get_cutoff();
    const double vol = e->boxLx * e->boxLy * e->boxLz;
    *e_lrc = -2.0 * M_PI * (double)n * (double)n / vol * csix / (3.0 * rc * rc * rc);
    *v_lrc = -2.0 * *e_lrc;
}

class GpuPath {
public:
    smd_ctx *ctx = nullptr;
    Ensemble *ens;
    std::vector<double> pos;    // 3 N doubles in Atom order: the current positions
    std::vector<double> sent;   // the last uploaded positions
    std::vector<double> frc;    // the forces of the last evaluation

    // precision: SMD_PREC_FP64 or SMD_PREC_MIXED; device: CUDA device index
    GpuPath(Ensemble *e, int precision = SMD_PREC_FP64, int device = 0) : ens(e) {
        SimConfiguration *cfg = e->myConfig;
        const int n = e->nAtoms;
        pos.assign(3 * (size_t)n, 0.0);
        frc.assign(3 * (size_t)n, 0.0);
        check(nullptr, smd_create(device, &ctx), "smd_create");
        std::vector<int32_t> type(n), mol(n);
        std::vector<double> mass(n), q(n);
        for (int i = 0; i < n; i++) {
            type[i] = e->atoms[i].atomType;
            mol[i] = e->atoms[i].molID;
            mass[i] = e->atoms[i].mass;
            q[i] = e->atoms[i].scaledCharge;
        }
        check(ctx, smd_set_topology(ctx, n, e->nAtomTypes, type.data(), mol.data(), mass.data(), q.data()),
              "smd_set_topology");
        // Ensemble::exclusionTable: per atom, partners up to a -1
        std::vector<int32_t> off(n + 1, 0), part;
        for (int i = 0; i < n; i++) {
            for (int k = 0; e->exclusionTable[i][k] != -1; k++) part.push_back(e->exclusionTable[i][k]);
            off[i + 1] = (int32_t)part.size();
        }
        if (part.empty()) part.push_back(0);
        check(ctx, smd_set_exclusions(ctx, off.data(), part.data()), "smd_set_exclusions");
        check(ctx, smd_set_box(ctx, e->boxLx, e->boxLy, e->boxLz), "smd_set_box");
        check(ctx, smd_set_pairlist(ctx, cfg->get_cutoff(), cfg->get_cutBuff(), e->useCellPairList ? 1 : 0),
              "smd_set_pairlist");
        if (cfg->compute_buffamoeba() || cfg->compute_multipol() || cfg->compute_wolf() ||
            cfg->compute_surf_correct())
            ERRORMSG("swinmd_gpu: this adapter carries the LJ and point-charge Ewald terms");
        // LJForce: sigma^2 and 4 eps per type pair (Parameters::set_lj_param)
        const int nt = e->nAtomTypes;
        std::vector<double> lj((size_t)nt * nt * 4, 0.0);
        for (int a = 0; a < nt; a++)
            for (int b = 0; b < nt; b++) {
                const LJPairParam p = e->myParams->get_lj_parameter(a, b);
                lj[4 * (a * nt + b)] = p.sigma;
                lj[4 * (a * nt + b) + 1] = p.eps;
            }
        double e_lrc = 0.0, v_lrc = 0.0;
        if (cfg->use_long_correct()) lj_tail(e, &e_lrc, &v_lrc);
        const double sd = cfg->get_switch_distance();
        check(ctx, smd_set_vdw(ctx, SMD_VDW_LJ, lj.data(), cfg->is_switch_on() ? 1 : 0, sd * sd, e_lrc, v_lrc),
              "smd_set_vdw");
        // EwaldForce: alpha, |k| cutoff and the real-space cutoff
        // (src/forces/EwaldForce.cpp:33-39)
        if (cfg->compute_ewald_force())
            check(ctx, smd_set_ewald(ctx, cfg->get_alpha(), cfg->get_k_cutoff(), cfg->get_cutoff()), "smd_set_ewald");
        // rigid molecules: the SHAKE distances of LFIntegrator::initialise
        // (src/integrators/LFIntegrator.cpp:141-167); they also tell the
        // library that the intramolecular corrections are energies only
        if (cfg->is_constraint_on()) {
            std::vector<double> len2(3 * (size_t)e->nMols, 0.0);
            for (int m = 0; m < e->nMols; m++) {
                Molecule &mol = e->molecules[m];
                if (mol.numAtoms < 2) continue;
                const int a0 = mol.myAtoms[0]->atomID, a1 = mol.myAtoms[1]->atomID;
                const double l01 = e->myParams->get_bond_length(a0, a1);
                len2[3 * m] = l01 * l01;
                if (mol.numAtoms >= 3) {
                    const int a2 = mol.myAtoms[2]->atomID;
                    const double l12 = e->myParams->get_bond_length(a1, a2);
                    const double l02 = e->myParams->get_bond_length(a0, a1, a2);
                    len2[3 * m + 1] = l12 * l12;
                    len2[3 * m + 2] = l02 * l02;
                } else {
                    len2[3 * m + 1] = len2[3 * m + 2] = len2[3 * m];
                }
            }
            check(ctx, smd_set_constraints(ctx, len2.data()), "smd_set_constraints");
        }
        check(ctx, smd_set_precision(ctx, precision), "smd_set_precision");
    }
    ~GpuPath() { smd_destroy(ctx); }

    // uploads the current positions when they changed since the last upload
    void sync_positions() {
        const int n = ens->nAtoms;
        for (int i = 0; i < n; i++) {
            const Vector3 &r = ens->atoms[i].position;
            pos[3 * i] = r.x;
            pos[3 * i + 1] = r.y;
            pos[3 * i + 2] = r.z;
        }
        if (sent.size() == pos.size() && std::memcmp(sent.data(), pos.data(), pos.size() * sizeof(double)) == 0)
            return;
        check(ctx, smd_upload_positions(ctx, pos.data()), "smd_upload_positions");
        sent = pos;
    }

    // evaluates `terms` at the current positions: forces into frc, energies
    // (SMD_E_COUNT) and the virial contribution (Ensemble::virial sign)
    void evaluate(uint32_t terms, double *energy, double *virial) {
        sync_positions();
        check(ctx, smd_compute_forces(ctx, terms, frc.data(), energy, virial), "smd_compute_forces");
    }

    // adds the forces of the last evaluation into Atom::force
    void add_forces() {
        for (int i = 0; i < ens->nAtoms; i++) {
            Vector3 &f = ens->atoms[i].force;
            f.x += frc[3 * i];
            f.y += frc[3 * i + 1];
            f.z += frc[3 * i + 2];
        }
    }
};

class GpuLJForce : public LJForce {
    GpuPath *path;

public:
    GpuLJForce(Ensemble *e, GpuPath *p) : LJForce(e), path(p) {}
    void compute() override {
        double en[SMD_E_COUNT], w[9];
        path->evaluate(SMD_TERM_VDW, en, w);
        path->add_forces();
        energy = en[SMD_E_VDW];
        myEnsemble->myEnergy.ljEnergy = energy;
        for (int k = 0; k < 9; k++) {
            virial[k] = -w[k];
            myEnsemble->virial[k] += w[k];
        }
    }
};

class GpuEwaldForce : public EwaldForce {
    GpuPath *path;

public:
    GpuEwaldForce(Ensemble *e, GpuPath *p) : EwaldForce(e), path(p) {}
    // real space, intramolecular correction, self and net-charge energies
    void compute() override {
        double en[SMD_E_COUNT], w[9];
        path->evaluate(SMD_TERM_EWALD_REAL, en, w);
        path->add_forces();
        myEnsemble->myEnergy.realEnergy = en[SMD_E_REAL];
        myEnsemble->myEnergy.correctEnergy = en[SMD_E_CORRECT];
        myEnsemble->myEnergy.molCorrectEnergy = en[SMD_E_MOLCORRECT];
        myEnsemble->myEnergy.surfCorrectEnergy = 0.0;
        energy = en[SMD_E_REAL] + en[SMD_E_CORRECT] + en[SMD_E_MOLCORRECT];
        for (int k = 0; k < 9; k++) {
            virial[k] = -w[k];
            myEnsemble->virial[k] += w[k];
        }
    }
    // reciprocal space: forces into Atom::force, as reciprocal_term adds them
    void compute_long() {
        double en[SMD_E_COUNT], w[9];
        path->evaluate(SMD_TERM_EWALD_LONG, en, w);
        path->add_forces();
        myEnsemble->myEnergy.longEnergy = en[SMD_E_LONG];
        for (int k = 0; k < 8; k++) myEnsemble->longVirial[k] = w[k];
    }
};

// The reference's LFIntegrator with its force objects on the GPU path.  Its
// constructor runs Integrator::initialise and LFIntegrator::start with the
// reference's own force objects; the GPU objects then take their place for
// every step of run().
class GpuForceLFIntegrator : public LFIntegrator {
public:
    GpuForceLFIntegrator(Ensemble *e, SimConfiguration *c, GpuPath *p) : LFIntegrator(e, c) {
        Force *old_lj = ljForce;
        ljForce = new GpuLJForce(e, p);
        for (Force *&f : forceGroup)
            if (f == old_lj) f = ljForce;
        delete old_lj;
        if (ewaldForce) {
            delete ewaldForce;
            ewaldForce = new GpuEwaldForce(e, p);
        }
    }
    double zeta() const { return fnh; }
    int list_updates() const { return numUpdates; }
};

}  // namespace swinmd_gpu

#endif
