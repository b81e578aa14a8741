/* swinmd_b200.h — C ABI of the B200 force + integration path for SwinMD.
 *
 * One opaque context holds one system on one GPU.  Every entry point returns
 * an int status (SMD_OK = 0) and never exits the process; the reference's
 * ERRORMSG/exit() paths (src/Errors.h:53-62) become non-zero codes, with the
 * message available from smd_last_error().  Arrays cross the boundary as
 * plain host pointers in the reference's layout: per-atom Vector3 values are
 * three consecutive doubles in atom order (Atom::position / velocity /
 * force, src/Atom.h:422-429); units are the reference's (nm, ps, amu,
 * kJ/mol, e; src/NEMD_defs.h:97-108).
 *
 * Each entry point names the reference interface it stands in for.
 */
#ifndef SWINMD_B200_H
#define SWINMD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct smd_ctx smd_ctx;

/* status codes */
enum {
    SMD_OK = 0,
    SMD_ERR_ARG = 1,          /* bad argument or call order */
    SMD_ERR_CUDA = 2,         /* a CUDA call failed */
    SMD_ERR_LIST_OVERFLOW = 3,/* a site has more neighbours than the list holds */
    SMD_ERR_NH_ITER = 4,      /* "NH iteration Error" (LFIntegrator.cpp:606-608) */
    SMD_ERR_SHAKE = 5,        /* SHAKE did not converge (LFIntegrator.cpp:1798-1812) */
    SMD_ERR_NAN = 6,          /* non-finite force or position */
    SMD_ERR_CG = 7,           /* dipole solve did not converge */
    SMD_ERR_NO_DEVICE = 8,    /* no CUDA device / extension unusable */
    SMD_ERR_TIMEOUT = 9,      /* a bounded device-side wait ran out (the dipole
                                 solve's grid barrier, see smd_set_wait_limit; the
                                 network's tensor-core completion wait) */
    SMD_ERR_BOX = 10          /* the barostat shrank the box below the cell grid's
                                 reach (run again from smd_integrator_start) */
};

/* arithmetic of the pair, reciprocal and dipole-field kernels */
enum {
    SMD_PREC_FP64 = 0,   /* FP64 math, 64-bit fixed-point accumulation */
    SMD_PREC_MIXED = 1   /* FP32 math on exact fixed-point displacements,
                            64-bit fixed-point accumulation */
};

/* force terms for smd_compute_forces (bit mask) */
enum {
    SMD_TERM_VDW = 1,        /* LJForce / MieForce / BMH pair term */
    SMD_TERM_EWALD_REAL = 2, /* EwaldForce::compute() real space + intra + self */
    SMD_TERM_EWALD_LONG = 4, /* EwaldForce::compute_long() */
    SMD_TERM_MP_SHORT = 8,   /* Multipole::compute(): self + real + intramolecular */
    SMD_TERM_MP_LONG = 16,   /* Multipole::compute_long() */
    SMD_TERM_IND_SHORT = 32, /* Induction::compute(): dipole solve, self, real, intra */
    SMD_TERM_IND_LONG = 64,  /* Induction::compute_long() (solves the dipoles if no
                                earlier call did for these positions) */
    SMD_TERM_BOND = 128,     /* BondForce::compute() */
    SMD_TERM_ANGLE = 256,    /* AngleForce::compute() */
    SMD_TERM_UB = 512,       /* UreyBradleyForce::compute() */
    SMD_TERM_WOLF = 1024,    /* WolfForce::compute() (energy into SMD_E_REAL) */
    SMD_TERM_ALL = 0xffff
};

/* energy components returned by smd_compute_forces, indices into energy[] */
enum {
    SMD_E_VDW = 0,       /* myEnergy.ljEnergy (incl. long-range correction) */
    SMD_E_REAL = 1,      /* myEnergy.realEnergy */
    SMD_E_LONG = 2,      /* myEnergy.longEnergy */
    SMD_E_CORRECT = 3,   /* myEnergy.correctEnergy (self + net charge) */
    SMD_E_MOLCORRECT = 4,/* myEnergy.molCorrectEnergy */
    SMD_E_SURF = 5,      /* myEnergy.surfCorrectEnergy */
    SMD_E_POL_REAL = 6,  /* myEnergy.realPolEnergy */
    SMD_E_POL_LONG = 7,  /* myEnergy.longPolEnergy */
    SMD_E_POL_SELF = 8,  /* myEnergy.correctPolEnergy */
    SMD_E_POL_INTRA = 9, /* myEnergy.molCorrectPolEnergy */
    SMD_E_POL_SURF = 10, /* myEnergy.surfacePolEnergy */
    SMD_E_BOND = 11,     /* myEnergy.bondEnergy */
    SMD_E_ANGLE = 12,    /* myEnergy.angleEnergy */
    SMD_E_UB = 13,       /* myEnergy.ubEnergy */
    SMD_E_TERMS = 14,    /* components summed into e_potential */
    SMD_E_COUNT = 16
};

/* vdW kinds for smd_set_vdw */
enum { SMD_VDW_NONE = 0, SMD_VDW_LJ = 1, SMD_VDW_MIE = 2, SMD_VDW_BMH = 3, SMD_VDW_BUFF = 4, SMD_VDW_SAAP = 5 };

/* initial guess of the induced-dipole solve (no reference counterpart: the
 * reference starts its CG from p = 1, src/forces/Induction.cpp:2401-2467) */
enum {
    SMD_GUESS_DIRECT = 0,      /* p0 = M^-1 E0: the preconditioner applied to the
                                  permanent field (alpha E0 with the site
                                  preconditioner) */
    SMD_GUESS_PREVIOUS = 1,    /* p0 = the previous solve's dipoles */
    SMD_GUESS_LEARNED = 2,     /* p0 = the extrapolated guess of order
                                  smd_mlp_set_base (default 2) + the per-site
                                  network's correction (smd_mlp_*) */
    SMD_GUESS_FIRST_ORDER = 3, /* p0 = p(t-1) + M^-1 (E0(t) - E0(t-1)): the learned
                                  guess of order 1 without the network */
    SMD_GUESS_EXTRAP2 = 4,     /* the mutual part u = p - M^-1 E0 extrapolated
                                  linearly over the stored steps:
                                  p0 = 2 p(t-1) - p(t-2)
                                       + M^-1 (E0(t) - 2 E0(t-1) + E0(t-2)) */
    SMD_GUESS_EXTRAP3 = 5      /* the same, quadratically:
                                  p0 = 3 p(t-1) - 3 p(t-2) + p(t-3)
                                       + M^-1 (E0(t) - 3 E0(t-1) + 3 E0(t-2) - E0(t-3)) */
};

/* thermostat kinds: SMD_THERMO_NOSE_HOOVER is the leap-frog integrator of
 * LFIntegrator; SMD_THERMO_NH_CHAIN selects the velocity-Verlet integrator
 * with the 4-link MTK chain of NHIntegrator::chain
 * (src/integrators/NHIntegrator.cpp:1814-1912) at constant volume, which
 * also carries SLLOD shear (strain_rate != 0, with Lees-Edwards images) */
enum { SMD_THERMO_NONE = 0, SMD_THERMO_NOSE_HOOVER = 1, SMD_THERMO_NH_CHAIN = 2 };

/* Leap-frog integrator settings: the config.txt fields that
 * LFIntegrator / Integrator read (src/Integrator.cpp:14-99). */
typedef struct {
    double timestep;       /* ps */
    double temperature;    /* K */
    double coupl_const;    /* Nose-Hoover tau (ps) */
    int thermostat;        /* SMD_THERMO_* */
    int atom_thermo;       /* 1: atomic kinetic energy drives zeta; 0: molecular */
    int constraint;        /* 0 none, 2 SHAKE (rigid 3-site water) */
    int long_steps;        /* reciprocal term every long_steps steps */
    double shake_tol;      /* SHAKE tolerance */
    int shake_max_iter;    /* SHAKE maxCount */
    int atom_ndf;          /* degrees of freedom (Integrator.cpp:22-27) */
    int mol_ndf;
    double strain_rate;    /* SLLOD planar Couette rate du_x/dy (1/ps); 0: equilibrium.
                              Needs SMD_THERMO_NH_CHAIN; takes the pair terms,
                              the point-charge Ewald sum (over the sheared cell's
                              k list, rebuilt on the device every evaluation)
                              and bonded terms, not multipoles, the buffered
                              14-7 or the surface correction */
} smd_integrator_params;

/* Per-step observables the reference keeps in Ensemble/Integrator members. */
typedef struct {
    int64_t step;            /* currentSteps */
    int64_t list_updates;    /* numUpdates */
    double energy[SMD_E_COUNT];
    double e_potential;      /* sum of energy[] (myEnergy.totEnergy without bonded terms) */
    double ke_atom;          /* myEnergy.atomKinEnergy = 0.5 sum m v^2 */
    double ke_mol;           /* myEnergy.molKinEnergy */
    double t_atom, t_mol;    /* atomTemp, molTemp (K) */
    double zeta;             /* fnh */
    double virial[9];        /* myEnsemble->virial (+ longVirial) */
    double atom_pressure[9]; /* Ensemble::atomPressure (kJ/mol/nm^3) */
    double mol_pressure[9];  /* Ensemble::molPressure */
    double volume;
    int64_t pairs_in_cutoff; /* unordered pairs inside the short-range cutoff */
    uint32_t status;
    uint32_t pad;
    double shear_offset;     /* Lees-Edwards offset of the images one box up (nm) */
} smd_observables;

/* Means over the steps since the last smd_averages_reset (or the context's
 * creation) of the observables Ensemble::accumulate averages
 * (src/Ensemble.cpp:814-894): energies and their squares, kinetic energies,
 * volume, and per pressure tensor (atomic, molecular) the stress figures
 * {pressure (trace / 3), shear (XY + YX) / 2, antisymmetric (YX - XY) / 2,
 * first normal difference XX - YY, second YY - ZZ} and the full tensor.
 * Every step of smd_run adds its sample on the device; smd_integrator_start
 * starts the sums afresh. */
typedef struct {
    int64_t samples;
    double e_potential, e_potential_sq, e_total, e_total_sq;
    double ke_atom, ke_atom_sq, ke_mol, ke_mol_sq, inv_ke_mol;
    double volume, volume_sq;
    double atom_stress[5], mol_stress[5];
    double atom_pressure[9], mol_pressure[9];
} smd_averages;

/* ---- lifetime -------------------------------------------------------- */
/* Creates a context on CUDA device `device` (the Simulation/Ensemble pair of
 * Simulation::setup_simulation, src/Simulation.cpp:171-263). */
int smd_create(int device, smd_ctx **out);
void smd_destroy(smd_ctx *ctx);
const char *smd_last_error(const smd_ctx *ctx);

/* ---- system (Ensemble::set_mol_system, src/Ensemble.cpp:140-227) ---- */
/* atom_type[n], mol_id[n], mass[n] (amu), scaled_charge[n] (charge times
 * SQRTCOULOMBCONSTANT, Atom::scaledCharge, src/Ensemble.cpp:183). */
int smd_set_topology(smd_ctx *ctx, int n_atoms, int n_types, const int32_t *atom_type,
                     const int32_t *mol_id, const double *mass, const double *scaled_charge);
/* Exclusion table (Ensemble::build_exclusion_table, src/Ensemble.cpp:323-367)
 * as CSR: partners of atom i are excl[offsets[i] .. offsets[i+1]). */
int smd_set_exclusions(smd_ctx *ctx, const int32_t *offsets, const int32_t *partners);
/* Box edges (Ensemble::boxLx..., src/Ensemble.cpp:370-420). */
int smd_set_box(smd_ctx *ctx, double lx, double ly, double lz);
/* Pair list (Ensemble::set_pairlist, src/Ensemble.cpp:454-473): list radius
 * cutoff + cut_buffer, cell list when use_cells and >= 3 cells per edge
 * (CellManager::set_cellManager, src/utils/CellManager.cpp:43-84). */
int smd_set_pairlist(smd_ctx *ctx, double cutoff, double cut_buffer, int use_cells);
/* Short-range pair term.  params: ntypes*ntypes rows of 4 doubles, meaning
 * per kind (LJ: sigma^2, 4 eps as Parameters::set_lj_param stores them,
 * src/Parameters.cpp:1360-1372; MIE: sigma, Cn*eps, n, m as MieForce derives
 * them, src/forces/MieForce.cpp:26-35,122-124; BMH: A, 1/rho, C, D).
 * LJ shifts the energy at the cutoff when switch_on (LJForce.cpp:152-168);
 * MIE and BMH apply the 5th-order switch from sqrt(switch_dist2) to the
 * cutoff (MieForce.cpp:145-154).  e_lrc/v_lrc: long-range correction energy
 * and virial added once per evaluation (LJForce.cpp:232-235). */
int smd_set_vdw(smd_ctx *ctx, int kind, const double *params, int switch_on,
                double switch_dist2, double e_lrc, double v_lrc);
/* Ewald summation for point charges (EwaldForce ctor + set_up,
 * src/forces/EwaldForce.cpp:22-257): alpha (1/nm), kcut (1/nm), real-space
 * cutoff.  long_steps: reciprocal term every long_steps steps. */
int smd_set_ewald(smd_ctx *ctx, double alpha, double kcut, double real_cut);
/* Buffered 14-7 pair term (BuffvdWForce, src/forces/BuffvdWForce.cpp):
 * params: ntypes*ntypes rows of {sigma, eps} as set_buff_param mixes them
 * (:392-433); n, m, delta, gamma; h_factor pulls type-0 (H) sites towards
 * their molecule's second site (O) (:358-385); taper c[6] from switch_dist
 * to the cutoff (:60-73); e_lrc / v_lrc the tail correction (:468-601). */
int smd_set_buff(smd_ctx *ctx, const double *params, double n, double m, double delta,
                 double gamma, double h_factor, int switch_on, double switch_dist,
                 const double *taper_c, double e_lrc, double v_lrc);
/* Bonded terms of flexible molecules (BondForce, AngleForce,
 * UreyBradleyForce; src/forces/BondForce.cpp:37-110, AngleForce.cpp:34-130,
 * UreyBradleyForce.cpp:39-100).  bonds[3*nbonds] = (atom1, atom2, type),
 * bond_params[2*type] = (r0 nm, k); angles[4*nangles] = (atom1, atom2 (the
 * apex), atom3, type), angle_params[2*type] = (theta0 rad, k).  form: 1
 * harmonic (U = k/2 d^2), 2 AMOEBA anharmonic (the reference's bendType 2:
 * quartic bond, sextic-in-degrees angle).  ub_on: the harmonic H-H term
 * k_ub (r - l0)^2 between the first and third site of every molecule.
 * nbonds = nangles = 0 and ub_on = 0 turn the terms off. */
int smd_set_bonded(smd_ctx *ctx, int nbonds, const int32_t *bonds, int nbond_types, const double *bond_params,
                   int nangles, const int32_t *angles, int nangle_types, const double *angle_params, int form,
                   int ub_on, double k_ub, double l0_ub);
/* Surface-dipole corrections (the surfCorrect option) of the point-charge
 * Ewald sum, the permanent multipoles and the induced dipoles
 * (EwaldForce::surfDipoleCorrect, src/forces/EwaldForce.cpp:816-937;
 * Multipole::surfDipoleCorrect, Multipole.cpp:1753-1920;
 * Induction::surfDipoleCorrect, Induction.cpp:2188-2380): evaluated with
 * SMD_TERM_EWALD_REAL, SMD_TERM_MP_SHORT and SMD_TERM_IND_SHORT as the
 * reference evaluates them inside those terms' compute(). */
int smd_set_surface_correct(smd_ctx *ctx, int on);
/* Polarisable multipole model (Multipole + Induction, src/forces/Multipole.cpp,
 * src/forces/Induction.cpp) for 3-site H O H molecules.  type_mp: per type
 * local-frame dipole (3) and traceless quadrupole (xx xy xz yy yz zz) as in
 * the !AtomParams section; polar: per type polarisability (nm^3); alpha,
 * kcut: Ewald splitting and |k| cutoff (1/nm); real_cut: cutoffEw;
 * induction: solve for induced dipoles; ind_cut: cutoffInd; thole_a. */
int smd_set_multipole(smd_ctx *ctx, const double *type_mp, const double *polar, double alpha,
                      double kcut, double real_cut, int induction, double ind_cut, double thole_a);
/* Dipole solver: RMS change tolerance (e nm), iteration cap, initial guess. */
int smd_set_solver(smd_ctx *ctx, double tol, int max_iter, int guess);
/* Preconditioner of the dipole solve.  No counterpart in the reference, which
 * runs unpreconditioned CG on its dense matrix (src/forces/Induction.cpp:
 * 2401-2467); the converged dipoles are the same, the iteration count is not.
 * SMD_PRECOND_SITE: diag(alpha_i).  SMD_PRECOND_MOLECULE (default): the
 * inverse of each molecule's own block of A (its sites' 1/alpha and their
 * Thole-damped mutual couplings), which also starts the solve from that
 * block solution under SMD_GUESS_DIRECT. */
#define SMD_PRECOND_SITE 0
#define SMD_PRECOND_MOLECULE 1
int smd_set_preconditioner(smd_ctx *ctx, int kind);
/* (no reference counterpart) Form of the solve with the molecule-block
 * preconditioner: mode 1 (the default) runs the pipelined PCG of Ghysels
 * and Vanroose (one grid barrier per iteration, w = A u and m = M^-1 w kept
 * by recurrence) in the mixed path, mode 2 in both precisions (in FP64 the
 * single-reduction form is the faster one), mode 0 never: the
 * single-reduction form of Chronopoulos and Gear (two barriers).  The same alpha, beta and stopping
 * test in exact arithmetic.  The pipelined form needs every molecule to be
 * three sites, molecule k's at sites 3k .. 3k + 2, and a tolerance of at
 * least 1e-9 e nm (its recurrences drift by rounding: on the polarisable
 * water it reaches 2e-10 and stalls near 1e-10); other
 * layouts and tighter tolerances use the single-reduction form. */
int smd_set_solver_pipelined(smd_ctx *ctx, int mode);
/* (no reference counterpart) Tensor-core path of the learned guess's
 * network (inference in the step and smd_mlp_eval): path 1 (the default)
 * runs the two hidden layers as 128-row tiles on the tcgen05 tensor cores
 * (BF16 operands in shared memory, FP32 accumulators in tensor memory),
 * path 0 as 16-row warp-level mma.sync tiles.  Both round the inputs and the
 * first hidden layer to BF16 and accumulate in FP32; their outputs agree to
 * FP32 summation order.  Training always uses the warp-level tiles. */
int smd_mlp_set_tensor_path(smd_ctx *ctx, int path);
/* Damping of the induced real-space energy, forces and torques, as the
 * reference's Config flag dampAmoeba selects (Induction.cpp:1051-1079):
 * form 0 (the default) multiplies the Ewald B_n by Thole's factors and skips
 * excluded pairs, form 1 is Tinker's AMOEBA form, which adds (1 - s l_n)
 * times the bare 1/r^n terms with the exclusion scale s inside, so excluded
 * pairs contribute.  The dipole solve is the same for both.  The mixed path
 * takes the unfused real-space kernels under form 1; smd_lustig refuses it. */
int smd_set_induction_damping(smd_ctx *ctx, int form);
/* Limit (seconds, default 1) of every bounded device-side wait: the dipole
 * solve's grid barrier.  A wait that runs out makes the solve leave, sets
 * SMD_ERR_TIMEOUT and keeps the context usable.  No reference counterpart
 * (the reference has no device waits). */
int smd_set_wait_limit(smd_ctx *ctx, double seconds);
/* Failure-path test hook, no reference counterpart: block `block` of the
 * following dipole solves returns before its first grid-barrier arrival, so
 * the other blocks' waits run out after the wait limit and the evaluation
 * returns SMD_ERR_TIMEOUT.  -1 (the default) turns it off. */
int smd_test_skip_arrival(smd_ctx *ctx, int block);
/* Solver statistics of the last solve: iterations and final RMS change. */
int smd_solver_stats(smd_ctx *ctx, int *iterations, double *rms_change);
/* RMS change of the dipoles at each iteration of the last solve (the
 * quantity the tolerance is tested on), up to 64 iterations: rms[k] for
 * k < min(count, cap).  The first entry measures how far the start was. */
int smd_solver_trace(smd_ctx *ctx, double *rms, int cap, int *count);
/* Lab-frame dipoles, quadrupoles, permanent field and induced dipoles of the
 * last evaluation, per site (each pointer may be NULL): mu[3n], quad[6n]
 * (xx xy xz yy yz zz, the reference's /3 convention), e0[3n], p[3n]. */
int smd_get_polarization(smd_ctx *ctx, double *mu, double *quad, double *e0, double *p);
/* Induced dipoles to start the next solve from (SMD_GUESS_PREVIOUS/LEARNED). */
int smd_set_induced(smd_ctx *ctx, const double *p);

/* ---- learned initial guess of the induced dipoles (no reference code) ----
 * The guess is the previous step's converged dipoles moved by the linear
 * response alpha (E0(t) - E0(t-1)) to the change of the permanent field
 * (each time step stores its dipoles and field; smd_integrator_start clears
 * the store), plus a correction from a per-site network (20 rotation-
 * invariant inputs in the site's own axes: the permanent fields at the
 * molecule's sites, the field change, the previous dipoles and their last
 * change; 2 hidden layers of 64, tanh).  The dipole solve then iterates from that guess to
 * the same tolerance.  Training rows are the solver's own converged dipoles. */
/* Allocates the network (seeded weights) and room for capacity_frames
 * configurations of training rows. */
int smd_mlp_init(smd_ctx *ctx, int capacity_frames, unsigned int seed);
/* The network's sizes: inputs per site (the width of smd_mlp_features and
 * smd_mlp_eval rows; smd_mlp_gradient rows add the 3 targets) and weights
 * (the gradient's length; smd_mlp_params adds 2 * features). */
int smd_mlp_dims(int *features, int *params);
/* Order (1-3) of the extrapolated guess the network corrects (SMD_GUESS_
 * FIRST_ORDER, EXTRAP2, EXTRAP3 without it).  Part of the trained model: set
 * it before smd_mlp_collect. */
int smd_mlp_set_base(smd_ctx *ctx, int order);
/* Appends the current configuration's rows (features and the converged
 * dipoles of the last force evaluation); needs two stored time steps. */
int smd_mlp_collect(smd_ctx *ctx);
/* Adam on the mean-squared error over all collected rows; *loss receives the
 * final error on one batch.  Marks the network ready for SMD_GUESS_LEARNED. */
int smd_mlp_train(smd_ctx *ctx, int epochs, int batch, double lr, unsigned int seed, double *loss);
/* Parameters (weights, then feature mean and 1/std): get and/or set;
 * *count receives their number. */
int smd_mlp_params(smd_ctx *ctx, float *get, const float *set, int *count);
/* Network output (3 per row) for raw feature rows (20 per row). */
int smd_mlp_eval(smd_ctx *ctx, const float *features, int rows, float *out);
/* Gradient of the batch loss for the given rows (20 features + 3 targets
 * each) at the current parameters; replaces the collected training rows. */
int smd_mlp_gradient(smd_ctx *ctx, const float *rows_data, int rows, float *grad);
/* Raw features (20 per site) of the current configuration, from the field
 * of the last evaluation. */
int smd_mlp_features(smd_ctx *ctx, float *features);
int smd_set_precision(smd_ctx *ctx, int mode);
/* FP64 path only.  on = 1: the buffered 14-7 with pow() as
 * BuffvdWForce::potFunc evaluates it (src/forces/BuffvdWForce.cpp:435-463)
 * and the multipole reciprocal sums with one FP64 sine and cosine of k.r per
 * (site, k) as Multipole::reciprocal_term and Induction::reciprocal_term do
 * (src/forces/Multipole.cpp:951-1245, src/forces/Induction.cpp:1395-1710).
 * on = 0 (default): the same quantities in FP64 by the algorithms the mixed
 * path uses (integer powers as products; the column passes with exact
 * 64-bit integer phases), which agree with the reference's forms to FP64
 * rounding.  No reference counterpart. */
int smd_set_reference_forms(smd_ctx *ctx, int on);
/* Pair-kernel threads per site (1..32, power of two); 0 lets the library pick. */
int smd_set_tuning(smd_ctx *ctx, int threads_per_site);

/* ---- state ------------------------------------------------------------ */
/* Positions pos[3 n].  Once a pair list exists (and without shear), the list
 * is kept while every site stays within half the skin of where it was at the
 * last rebuild, minimum image, the same test a step makes; otherwise the next
 * step rebuilds it.  A non-finite coordinate returns SMD_ERR_NAN and leaves
 * the state unchanged (the reference would carry it into every force). */
int smd_upload_positions(smd_ctx *ctx, const double *pos);
/* vel: Atom::velocity; vtminus may be NULL (then set by smd_integrator_start) */
int smd_upload_velocities(smd_ctx *ctx, const double *vel, const double *vtminus);
int smd_download_state(smd_ctx *ctx, double *pos, double *vel, double *vtminus);
/* Atom::realPos, the positions without the periodic wraps (written to
 * state.out by Integrator::write_state, src/Integrator.cpp:275-302): the
 * positions less the box shifts each molecule has had since the last
 * smd_upload_positions, plus the offsets an smd_upload_real_positions after
 * that upload set (a restart's realPos). */
int smd_download_real_positions(smd_ctx *ctx, double *real);
int smd_upload_real_positions(smd_ctx *ctx, const double *real);
/* The integrator's scalars (32 doubles: the Nose-Hoover zeta and its
 * half-step value, the pending centre-of-mass correction, the chain
 * velocities, the Lees-Edwards offset), for a restart that continues the
 * trajectory where a checkpoint left it (the reference restarts with zeta
 * = 0: Ensemble::set_configuration, src/Ensemble.cpp:303-317). */
int smd_get_integrator_state(smd_ctx *ctx, double *state);
int smd_set_integrator_state(smd_ctx *ctx, const double *state);

/* ---- forces (Force::compute / compute_long, src/Force.h:59) ----------
 * Evaluates the selected terms at the current positions and returns:
 * force[3n] (the terms' contribution to Atom::force), energy[SMD_E_COUNT]
 * (NULL allowed), virial[9] (contribution to Ensemble::virial + longVirial,
 * i.e. +sum r_ij f_ij; NULL allowed).  As in the reference's step, the pair
 * list is rebuilt only once a site has moved half the skin since the last
 * build (src/integrators/LFIntegrator.cpp:307-341), and the induced dipoles
 * are solved once per configuration: SMD_TERM_IND_LONG after
 * SMD_TERM_IND_SHORT on the same positions uses the dipoles that call solved,
 * as Induction::compute_long uses those of Induction::compute.  The device
 * output buffer is allocated on the first call and kept with the context. */
int smd_compute_forces(smd_ctx *ctx, uint32_t terms, double *force, double *energy,
                       double *virial);
/* Unordered pairs of the current Verlet list as (i < j) int32 pairs, the set
 * CellManager::update_pair_list builds (src/utils/CellManager.cpp:216-314).
 * cap: room in pairs[] for `cap` pairs; *count receives the number found. */
int smd_get_pairs(smd_ctx *ctx, int32_t *pairs, int64_t cap, int64_t *count);
/* smd_compute_forces for callers that may not allocate device memory (a
 * host loop with a fixed memory budget, a process that must not call
 * cudaMalloc after set-up): the same evaluation and results, with the device
 * force buffer taken from a static array of 65536 x 3 doubles inside the
 * library instead of the context's own buffer (which smd_compute_forces
 * allocates on its first call).  No reference counterpart (the reference
 * evaluates forces on the host).  Returns SMD_ERR_ARG for systems of more
 * than 65536 sites.  Calls that overlap on one device (threads, or several
 * contexts) share the array and race.  The first call on a device resolves
 * the array's address (cudaGetSymbolAddress) with that device current, under
 * a lock; make that first call outside any stream capture.  The address is
 * forgotten when the device's last context is destroyed: after a device
 * reset, destroy that device's contexts before creating new ones. */
int smd_compute_forces_noalloc(smd_ctx *ctx, uint32_t terms, double *force, double *energy, double *virial);
/* k-vector count of the Ewald reciprocal set (EwaldForce::set_up). */
int smd_ewald_nk(smd_ctx *ctx, int *nk);

/* ---- integration (LFIntegrator, src/integrators/LFIntegrator.cpp) ------ */
int smd_set_integrator(smd_ctx *ctx, const smd_integrator_params *p);
/* Isotropic barostat of the reference's NpT run (NHIntegrator with
 * ensemble 1, src/integrators/NHIntegrator.cpp:276-694, chain :1814-1912):
 * the chain integrator (SMD_THERMO_NH_CHAIN) then carries vlog with mass
 * W = (Nf + 1) kT BarosConst^2 and scales positions and box each step.
 * pressure is the config's value (divided by 1.66053904042716 into
 * kJ/mol/nm^3 as Integrator.cpp:44 does).  The barostat reads the virial
 * pressure as the reference does with computeLustig on.  Pair terms
 * (LJ, Mie, Buckingham) in FP64 only, without constraints; other set-ups
 * are refused at smd_integrator_start.  on = 0 switches it off. */
/* Wolf summation of the point charges instead of Ewald (WolfForce,
 * src/forces/WolfForce.cpp:100-260; computeWolf): every listed pair within
 * the cutoff adds q_i q_j (erfc(a r)/r - erfc(a rc)/rc) to the energy and
 * the force factor shifted by its value at the cutoff.  msite (n entries,
 * or null): 1 where a site's charge sits on the displaced site of
 * WolfForce::DummyPosition (the reference flags the type-1 site of every
 * "WAT" molecule), d_op its distance from the molecule's second site in nm
 * (R_OP over F_Length in the reference).  The charge term then runs as a
 * second FP64 pass; without displaced sites it is fused into the pair pass. */
/* SAAP pair potential (SAAPForce::compute, src/forces/SAAPForce.cpp:54-230)
 * as the vdW term: U = (a0 e^(a1 r)/r + a2 e^(a3 r) + a4) / (1 + a5 r^6)
 * between sites of different molecules within the cutoff, with the
 * reference's 5th-order switch as SAAPForce applies it.  table: ntypes^2
 * rows of (a0, a1, a2, a3, a4, a5).  No tail correction (the reference's is
 * for its three-type CO2 table only). */
/* Lustig's volume derivatives of the LJ term at the current positions
 * (LJForce::compute with computeLustig: Ensemble::myLustig.ljUlus, ljdUlus,
 * ljd2Ulus, src/forces/LJForce.cpp:136-150, 230-247): out[0] = U, out[1] =
 * dU/dV, out[2] = d2U/dV2, tail correction included; under constraints the
 * pair term takes r_ij . R_ij with R_ij the molecules' centre difference. */
int smd_lustig_lj(smd_ctx *ctx, double *out);
/* Every field of Ensemble::myLustig (src/Ensemble.h:77-108) at the current
 * configuration, as the reference's force terms write them during a step:
 * the LJ (LJForce.cpp:136-250) or buffered 14-7 (BuffvdWForce.cpp:244-335)
 * values, the point-charge Ewald sums' real, intramolecular, surface and
 * reciprocal derivatives (EwaldForce.cpp:129-192, 405-411, 596-675,
 * 770-790, 850-863), the multipoles' (Multipole.cpp:163-240 with the torque
 * mapping's dU/dV, :1946-2134), the induced dipoles' (Induction.cpp:486-590),
 * and bonds and Urey-Bradley (BondForce.cpp:86-105,
 * UreyBradleyForce.cpp:76-95).  Positions with constraints use the
 * molecules' centres of mass as the reference does (r_ij . R_ij and the
 * reciprocal centre-of-mass sums).  Evaluated in FP64 whatever the precision
 * mode; the induced dipoles are solved at the solver's settings first.
 * out[SMD_LUSTIG_COUNT] in the struct's order (SMD_LUS_*); fields no term
 * writes (inducEn, inducDeriv, intravirPolCorrect, the second derivatives
 * the reference leaves at zero) come back 0, and so does virialcorrect,
 * which LFIntegrator forms after the position update from one step's forces
 * and the next step's positions (LFIntegrator.cpp:819-836).  The Wolf sum's
 * realDeriv/realSecDeriv follow WolfForce.cpp:200-244.  Refused
 * (SMD_ERR_ARG) with Mie, BMH or SAAP pair terms and in a sheared cell. */
enum {
    SMD_LUS_LJ_U = 0, SMD_LUS_LJ_DU, SMD_LUS_LJ_D2U, SMD_LUS_VIRCORRECT, SMD_LUS_INTRAVIR,
    SMD_LUS_LONG, SMD_LUS_REAL, SMD_LUS_REAL2, SMD_LUS_LONG2, SMD_LUS_SURF, SMD_LUS_SURF2,
    SMD_LUS_INDUC_EN, SMD_LUS_INDUC, SMD_LUS_MOL, SMD_LUS_MOL2, SMD_LUS_BOND, SMD_LUS_BOND2,
    SMD_LUS_POL_INTRAVIR, SMD_LUS_POL_LONG, SMD_LUS_POL_REAL, SMD_LUS_POL_REAL2, SMD_LUS_POL_LONG2,
    SMD_LUS_POL_SURF, SMD_LUS_POL_SURF2, SMD_LUS_POL_MOL, SMD_LUS_POL_MOL2, SMD_LUS_POL_SELF,
    SMD_LUS_UB, SMD_LUS_UB2, SMD_LUSTIG_COUNT
};
int smd_lustig(smd_ctx *ctx, double *out);
int smd_set_saap(smd_ctx *ctx, const double *table, int switch_on, double switch_dist2);
int smd_set_wolf(smd_ctx *ctx, double alpha, double cutoff, const int *msite, double d_op);
int smd_set_barostat(smd_ctx *ctx, double pressure, double baros_const, int on);
/* Current box edges (the barostat's, when it runs). */
int smd_get_box(smd_ctx *ctx, double *edges);
/* SHAKE targets (LFIntegrator::initialise, LFIntegrator.cpp:141-167):
 * len2[3*m + k] = squared length of the k-th cyclic distance of molecule m
 * (sites 0-1, 1-2, 2-0 of a 3-site molecule; 0-1, 1-2 of a chain). */
int smd_set_constraints(smd_ctx *ctx, const double *len2);
/* LFIntegrator::start (LFIntegrator.cpp:991-1174): F(0) and
 * vtMinus = v - dt/2 F/m. */
int smd_integrator_start(smd_ctx *ctx);
/* smd_integrator_start without LFIntegrator::start's half-step velocities:
 * the velocities and vtMinus uploaded by smd_upload_velocities are kept, as
 * the reference's run that does not start new takes them from state.in and
 * vtMinus.in (LFIntegrator.cpp:187-192).  The chain integrator's scalars are
 * reset as by smd_integrator_start; smd_set_integrator_state afterwards
 * restores the saved ones. */
int smd_integrator_resume(smd_ctx *ctx);
/* LFIntegrator::run(nsteps) (LFIntegrator.cpp:252-942) without file output. */
int smd_run(smd_ctx *ctx, int nsteps);
int smd_get_observables(smd_ctx *ctx, smd_observables *out);
/* Per-step samples recorded during smd_run (e_potential, ke_atom, t_atom, zeta,
 * atom-pressure trace/3) for the last min(nsteps, cap) steps: out[5*cap]. */
int smd_set_series_capacity(smd_ctx *ctx, int cap);
int smd_get_series(smd_ctx *ctx, double *out, int cap, int *count);

/* ---- observables on the device ----------------------------------------- */
int smd_averages_reset(smd_ctx *ctx);
int smd_get_averages(smd_ctx *ctx, smd_averages *out);
/* Radial distribution function (RDF, src/observables/RDF.cpp): histogram of
 * every non-excluded pair closer than the smallest half box edge, per type
 * pair, nbins bins.  Setup clears it; each sample adds the current
 * configuration (RDF::sampling, :109-144). */
int smd_rdf_setup(smd_ctx *ctx, int nbins);
int smd_rdf_sample(smd_ctx *ctx);
/* hist[ntypes][ntypes][nbins] raw counts (both type orders of every pair;
 * may be NULL); g[npairs][nbins] the normalised RDF of each type pair
 * t1 <= t2 in the order of RDF::write_result (:146-180; may be NULL);
 * r_mid[nbins] the bin centres (may be NULL); *samples the samples taken. */
int smd_rdf_get(smd_ctx *ctx, uint64_t *hist, double *g, double *r_mid, int64_t *samples);

/* ---- measurement ------------------------------------------------------- */
/* Average device time (ms, CUDA events on the context's stream) of each
 * stage of one step, each launched `reps` times on its own:
 * out[0] pair kernel, out[1] reciprocal kernels, out[2] integrate kernel,
 * out[3] a forced pair-list rebuild; for the polarisable model out[4] frames,
 * out[5] multipole real+self+intra, out[6] multipole reciprocal (models
 * without induced dipoles), out[7] field + dipole solve, out[8] induced
 * real+self+intra (in the mixed precision mode the multipole and induced
 * real space are one fused pass after the solve: out[8] then holds both and
 * out[5] is 0), out[9] reciprocal structure factors and forces of the
 * permanent and induced multipoles together, out[10] the permanent field
 * with the solve's tensor rows, preconditioner blocks and start dipoles,
 * out[11] the PCG kernel alone (out has room for 12).  Leaves forces and
 * state unchanged except for the rebuilt list. */
int smd_profile_stages(smd_ctx *ctx, int reps, double *out);
/* smd_run with the device time of the nsteps graph launches (CUDA events on
 * the context's stream, synchronized on both sides) returned in *device_ms. */
int smd_run_timed(smd_ctx *ctx, int nsteps, double *device_ms);
/* Number of kernel launches in one step of smd_run (kernel nodes of the
 * step's CUDA graph). */
int smd_step_kernel_count(smd_ctx *ctx, int *count);

/* ---- batched replicas ---------------------------------------------------- */
/* Many independent systems (replicas of uneven size, each with its own
 * seed, strain rate and thermostat chain) advanced together: one CUDA graph
 * per step whose branches are the replicas' steps, each on its replica's
 * stream, so one launch runs them all concurrently on the device.  The
 * reference runs such replicas as separate processes (one Simulation per
 * run, src/NEMDMain.cpp); there is no reference interface for the batch
 * itself.  The contexts must be on one device with their integrators set
 * and started; they stay owned by the caller and must outlive the batch,
 * and must not be reconfigured while it exists. */
typedef struct smd_batch smd_batch;
int smd_batch_create(smd_ctx *const *ctxs, int count, smd_batch **out);
void smd_batch_destroy(smd_batch *batch);
const char *smd_batch_last_error(const smd_batch *batch);
/* Autotuner: for each replica, times its pair kernel `reps` times at every
 * threads-per-site shape (1, 2, ..., 32), keeps the fastest (tpp_out[r], may
 * be null) and recomputes the replica's forces. */
int smd_batch_autotune(smd_batch *batch, int reps, int32_t *tpp_out);
/* nsteps steps of every replica; *device_ms (may be null) gets the device
 * time of the graph launches (CUDA events on the batch stream). */
int smd_batch_run(smd_batch *batch, int nsteps, double *device_ms);

#ifdef __cplusplus
}
#endif
#endif
