// swinmd_gpu.h -- the C++ adapter that puts SwinMD's force terms on the B200
// path, through the C ABI of libswinmd_b200.so (include/swinmd_b200.h).
//
// It sits beside the reference's own classes and changes none of them:
//
//   GpuPath                one smd_ctx per Ensemble, set up from the
//                          reference's Ensemble / Parameters /
//                          SimConfiguration objects (Simulation::setup_simulation,
//                          src/Simulation.cpp:171-263)
//   GpuNonbonded<Base>     every non-bonded term the configuration enables
//                          (LJForce or BuffvdWForce, EwaldForce or Multipole +
//                          Induction, their surface terms), evaluated in two
//                          calls per step (short range, reciprocal space),
//                          standing in the slot of Base = LJForce or
//                          BuffvdWForce, the one force object
//                          LFIntegrator::run always calls
//                          (src/integrators/LFIntegrator.cpp:387-400)
//   GpuForceLFIntegrator   the reference's own LFIntegrator (leap-frog,
//                          Nose-Hoover, SHAKE, bonded terms on the host)
//                          driving it: the vdW pointer Integrator::initialise
//                          filled (src/Integrator.cpp:111-203) is swapped for
//                          the GPU object and the electrostatic branches of
//                          LFIntegrator::run (:411-458) are switched off, as
//                          the GPU object already computed those terms.
//                          (EwaldForce::compute_long, Multipole::compute_long
//                          and Induction::compute_long are not virtual, so a
//                          derived object in their slots would not be called.)
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
#include "forces/BuffvdWForce.h"
#include "forces/EwaldForce.h"
#include "forces/Induction.h"
#include "forces/LJForce.h"
#include "forces/Multipole.h"

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

// BuffvdWForce::set_buff_param (src/forces/BuffvdWForce.cpp:392-433): per
// type pair the cubic-mean sigma and the HHG epsilon; a pair with a zero
// epsilon gets sigma 1e-7 and epsilon 0.  tab: nt * nt * 2 (sigma, eps).
inline void buff_table(Ensemble *e, std::vector<double> &tab) {
    const int nt = e->nAtomTypes;
    tab.assign((size_t)nt * nt * 2, 0.0);
    for (int a = 0; a < nt; a++)
        for (int b = 0; b < nt; b++) {
            const AtomParam &pa = e->myParams->atomParams[a], &pb = e->myParams->atomParams[b];
            double *t = &tab[2 * (a * nt + b)];
            if (pa.eps == 0.0 || pb.eps == 0.0) {
                t[0] = 0.0000001;
                t[1] = 0.0;
                continue;
            }
            const double si2 = pa.sigma * pa.sigma, sj2 = pb.sigma * pb.sigma;
            const double es = std::sqrt(pa.eps) + std::sqrt(pb.eps);
            t[0] = (si2 * pa.sigma + sj2 * pb.sigma) / (si2 + sj2);
            t[1] = (4.0 * pa.eps * pb.eps) / (es * es);
        }
}

// BuffvdWForce::potFunc (BuffvdWForce.cpp:435-463): energy and dU/dr
inline void buff_pot(double r, double sigma, double eps, double n, double m, double delta, double gamma,
                     double &u, double &f) {
    if (eps == 0.0) { u = f = 0.0; return; }
    const double inv = 1.0 / sigma, rho = r * inv;
    const double rho_m = std::pow(rho, m), rho_m1 = std::pow(rho, m - 1.0), nm = n - m;
    const double par1 = (1.0 + delta) / (rho + delta), par2 = (1.0 + gamma) / (rho_m + gamma);
    const double p1 = std::pow(par1, nm);
    u = eps * p1 * (par2 - 2.0);
    f = -eps * nm * p1 * (par2 - 2.0) * inv / (rho + delta) - eps * p1 * par2 * m * rho_m1 * inv / (rho_m + gamma);
}

// BuffvdWForce::long_range_correct (BuffvdWForce.cpp:468-601): the trapezoid
// rule with 2^20 intervals of r^2 U and r^3 U' from the cutoff to 5000 nm,
// averaged over the type pairs of all atoms
inline void buff_tail(Ensemble *e, const std::vector<double> &tab, double *e_lrc, double *v_lrc) {
    SimConfiguration *c = e->myConfig;
    const int nt = e->nAtomTypes, n = e->nAtoms;
    std::vector<long long> count(nt, 0);
    for (int i = 0; i < n; i++) count[e->atoms[i].atomType]++;
    const double rc = c->get_cutoff(), vol = e->boxLx * e->boxLy * e->boxLz;
    const double nb = c->get_nBuff_param(), mb = c->get_mBuff_param();
    const double db = c->get_deltaBuff_param(), gb = c->get_gammaBuff_param();
    const long long intervals = 1LL << 20;
    const double h = (5000.0 - rc) / (double)intervals;
    double U = 0.0, P = 0.0;
    long long npair = 0;
    for (int a = 0; a < nt; a++)
        for (int b = a; b < nt; b++) {
            const long long nij = a != b ? count[a] * count[b] : (long long)(count[a] * (count[a] - 1) * 0.5);
            npair += nij;
            const double sig = tab[2 * (a * nt + b)], eps = tab[2 * (a * nt + b) + 1];
            double u, f;
            buff_pot(rc, sig, eps, nb, mb, db, gb, u, f);
            double su = 0.5 * h * rc * rc * u, sp = 0.5 * h * rc * rc * rc * f;
            for (long long k = 1; k < intervals; k++) {
                const double r = rc + (double)k * h;
                buff_pot(r, sig, eps, nb, mb, db, gb, u, f);
                su += h * r * r * u;
                sp += h * r * r * r * f;
            }
            buff_pot(5000.0, sig, eps, nb, mb, db, gb, u, f);
            su += 0.5 * h * 5000.0 * 5000.0 * u;
            sp += 0.5 * h * 5000.0 * 5000.0 * 5000.0 * f;
            U += (double)nij * su;
            P += (double)nij * sp;
        }
    if (npair <= 0) { *e_lrc = *v_lrc = 0.0; return; }
    U /= (double)npair;
    P /= (double)npair;
    *e_lrc = 2.0 * M_PI * (double)n * (double)n / vol * U;
    *v_lrc = 2.0 * M_PI * (double)n * (double)n / (vol * vol) * P / 3.0 * vol;
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
        if (cfg->compute_wolf())
            ERRORMSG("swinmd_gpu: this adapter carries LJ, buffered 14-7, Ewald and the multipole model");
        // molecule kinds with their own branches in the electrostatic terms
        // (the dummy charge site of "MCY", the damping of "BBV")
        for (int m = 0; m < e->nMols; m++)
            if (!std::strcmp(e->molecules[m].molName, "MCY") || !std::strcmp(e->molecules[m].molName, "BBV"))
                ERRORMSG("swinmd_gpu: MCY and BBV molecules are not built on the GPU path");
        const int nt = e->nAtomTypes;
        const double sd = cfg->get_switch_distance();
        if (cfg->compute_buffamoeba()) {
            // BuffvdWForce: mixed table, taper from the switch distance to
            // the cutoff (BuffvdWForce.cpp:60-73), tail correction
            std::vector<double> tab;
            buff_table(e, tab);
            const double rc = cfg->get_cutoff(), rc2 = rc * rc, sd2 = sd * sd, off = rc - sd;
            const double den = off * off * off * off * off;
            const double taper[6] = {rc * rc2 * (rc2 - 5.0 * rc * sd + 10.0 * sd2) / den, -30.0 * rc2 * sd2 / den,
                                     30.0 * (rc2 * sd + rc * sd2) / den, -10.0 * (rc2 + 4.0 * rc * sd + sd2) / den,
                                     15.0 * (rc + sd) / den, -6.0 / den};
            double e_lrc = 0.0, v_lrc = 0.0;
            if (cfg->use_long_correct()) buff_tail(e, tab, &e_lrc, &v_lrc);
            check(ctx, smd_set_buff(ctx, tab.data(), cfg->get_nBuff_param(), cfg->get_mBuff_param(),
                                    cfg->get_deltaBuff_param(), cfg->get_gammaBuff_param(),
                                    cfg->get_hfactor_reduction(), cfg->is_switch_on() ? 1 : 0, sd, taper, e_lrc,
                                    v_lrc),
                  "smd_set_buff");
        } else {
            // LJForce: sigma^2 and 4 eps per type pair (Parameters::set_lj_param)
            std::vector<double> lj((size_t)nt * nt * 4, 0.0);
            for (int a = 0; a < nt; a++)
                for (int b = 0; b < nt; b++) {
                    const LJPairParam p = e->myParams->get_lj_parameter(a, b);
                    lj[4 * (a * nt + b)] = p.sigma;
                    lj[4 * (a * nt + b) + 1] = p.eps;
                }
            double e_lrc = 0.0, v_lrc = 0.0;
            if (cfg->use_long_correct()) lj_tail(e, &e_lrc, &v_lrc);
            check(ctx, smd_set_vdw(ctx, SMD_VDW_LJ, lj.data(), cfg->is_switch_on() ? 1 : 0, sd * sd, e_lrc, v_lrc),
                  "smd_set_vdw");
        }
        if (cfg->compute_multipol()) {
            // Multipole / Induction: per type local-frame dipole, quadrupole
            // and polarisability (Parameters' AtomParam), Ewald and
            // induction cutoffs, Thole a; the dipoles solved far below the
            // reference's own stopping point (|r| < 1e-14)
            std::vector<double> mpv((size_t)nt * 9), pol(nt);
// (NccForce.h defines a macro named after AtomParam's polarisability field)
#pragma push_macro("polar")
#undef polar
            for (int t = 0; t < nt; t++) {
                const AtomParam &ap = e->myParams->atomParams[t];
                const double v[9] = {ap.dipx, ap.dipy, ap.dipz, ap.quadxx, ap.quadxy, ap.quadxz,
                                     ap.quadyy, ap.quadyz, ap.quadzz};
                for (int k = 0; k < 9; k++) mpv[9 * t + k] = v[k];
                pol[t] = ap.polar;
            }
#pragma pop_macro("polar")
            check(ctx, smd_set_multipole(ctx, mpv.data(), pol.data(), cfg->get_alpha(), cfg->get_k_cutoff(),
                                         cfg->get_cutoffEw(), cfg->compute_induction() ? 1 : 0,
                                         cfg->get_cutoffInd(), cfg->get_adamping()),
                  "smd_set_multipole");
            check(ctx, smd_set_solver(ctx, 1e-13, 3000, SMD_GUESS_DIRECT), "smd_set_solver");
        }
        if (cfg->compute_surf_correct()) check(ctx, smd_set_surface_correct(ctx, 1), "smd_set_surface_correct");
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

    // Ensemble::myLustig as the replaced classes leave it after a step's
    // force calls (smd_lustig, FP64): the electrostatic fields every step
    // (EwaldForce, Multipole and Induction write theirs unconditionally), the
    // buffered 14-7's U and dU/dV every step and its d2U/dV2 with
    // computeLustig (BuffvdWForce.cpp:326-336), the LJ fields with
    // computeLustig only (LJForce.cpp:136-250).  The bonded fields belong to
    // the host's own BondForce / UreyBradleyForce and virialcorrect to the
    // integrator; they are left alone.  `lustig = false` skips the
    // evaluation (the fields then keep their last values).
    bool lustig = true;
    void fill_lustig(bool compute_lustig, bool buff) {
        static_assert(sizeof(Lustig) == SMD_LUSTIG_COUNT * sizeof(double), "Lustig layout");
        double v[SMD_LUSTIG_COUNT];
        sync_positions();
        check(ctx, smd_lustig(ctx, v), "smd_lustig");
        double *L = reinterpret_cast<double *>(&ens->myLustig);
        for (int q = 0; q < SMD_LUSTIG_COUNT; q++) {
            if (q == SMD_LUS_VIRCORRECT || q == SMD_LUS_BOND || q == SMD_LUS_BOND2 || q == SMD_LUS_UB ||
                q == SMD_LUS_UB2)
                continue;
            if (q == SMD_LUS_LJ_U || q == SMD_LUS_LJ_DU || q == SMD_LUS_LJ_D2U) {
                const bool always = buff && q != SMD_LUS_LJ_D2U;
                if (!always && !compute_lustig) continue;
            }
            L[q] = v[q];
        }
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

// The non-bonded terms of the step in the slot of Base (LJForce or
// BuffvdWForce).  Forces add into Atom::force; energies are assigned into the
// myEnergy fields the replaced classes assign; the short-range virial goes
// into Ensemble::virial with the reference's sign, and the reciprocal virial
// into Ensemble::longVirial components 0..7, as EwaldForce::compute_long and
// Multipole::compute_long + Induction::compute_long leave them.
template <class Base>
class GpuNonbonded : public Base {
    GpuPath *path;
    uint32_t short_terms = SMD_TERM_VDW, long_terms = 0;

public:
    GpuNonbonded(Ensemble *e, GpuPath *p) : Base(e), path(p) {
        SimConfiguration *c = e->myConfig;
        if (c->compute_ewald_force()) {
            short_terms |= SMD_TERM_EWALD_REAL;
            long_terms |= SMD_TERM_EWALD_LONG;
        } else if (c->compute_multipol()) {
            short_terms |= SMD_TERM_MP_SHORT;
            long_terms |= SMD_TERM_MP_LONG;
            if (c->compute_induction()) {
                short_terms |= SMD_TERM_IND_SHORT;
                long_terms |= SMD_TERM_IND_LONG;
            }
        }
    }
    void compute() override {
        double en[SMD_E_COUNT], w[9];
        Energy &E = this->myEnsemble->myEnergy;
        path->evaluate(short_terms, en, w);
        path->add_forces();
        this->energy = en[SMD_E_VDW];
        E.ljEnergy = en[SMD_E_VDW];   // tail correction included
        if (short_terms & (SMD_TERM_EWALD_REAL | SMD_TERM_MP_SHORT)) {
            E.realEnergy = en[SMD_E_REAL];
            E.correctEnergy = en[SMD_E_CORRECT];
            E.molCorrectEnergy = en[SMD_E_MOLCORRECT];
            E.surfCorrectEnergy = en[SMD_E_SURF];
        }
        if (short_terms & SMD_TERM_IND_SHORT) {
            E.realPolEnergy = en[SMD_E_POL_REAL];
            E.correctPolEnergy = en[SMD_E_POL_SELF];
            E.molCorrectPolEnergy = en[SMD_E_POL_INTRA];
            E.surfacePolEnergy = en[SMD_E_POL_SURF];
        }
        for (int k = 0; k < 9; k++) {
            this->virial[k] = -w[k];
            this->myEnsemble->virial[k] += w[k];
        }
        if (long_terms) {
            path->evaluate(long_terms, en, w);
            path->add_forces();
            E.longEnergy = en[SMD_E_LONG];
            if (long_terms & SMD_TERM_IND_LONG) E.longPolEnergy = en[SMD_E_POL_LONG];
            for (int k = 0; k < 8; k++) this->myEnsemble->longVirial[k] = w[k];
        }
        if (path->lustig)
            path->fill_lustig(this->myEnsemble->myConfig->compute_lustig(),
                              this->myEnsemble->myConfig->compute_buffamoeba());
    }
};

// The reference's LFIntegrator with its force objects on the GPU path.  Its
// constructor runs Integrator::initialise and LFIntegrator::start with the
// reference's own force objects; the GPU objects then take their place for
// every step of run().
class GpuForceLFIntegrator : public LFIntegrator {
public:
    GpuForceLFIntegrator(Ensemble *e, SimConfiguration *c, GpuPath *p) : LFIntegrator(e, c) {
        if (buffForce) {
            Force *old = buffForce;
            buffForce = new GpuNonbonded<BuffvdWForce>(e, p);
            for (Force *&f : forceGroup)
                if (f == old) f = buffForce;
            delete old;
        } else {
            Force *old = ljForce;
            ljForce = new GpuNonbonded<LJForce>(e, p);
            for (Force *&f : forceGroup)
                if (f == old) f = ljForce;
            delete old;
        }
        // the GPU object computes the electrostatic terms too
        computeEwald = false;
        computeMultipole = false;
        computeInduction = false;
    }
    double zeta() const { return fnh; }
    // the step's Lustig pressure (LFIntegrator.cpp:731-741)
    double lustig_pressure() const { return molPt; }
    int list_updates() const { return numUpdates; }
};

}  // namespace swinmd_gpu

#endif
