// Host-side context of one simulated system and the launchers of its kernels.
// The C-ABI in include/swinmd_b200.h hands callers an opaque pointer to this.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include "smd_common.cuh"
#include "../../include/swinmd_b200.h"

namespace smd {

enum VdwKind { VDW_NONE = 0, VDW_LJ = 1, VDW_MIE = 2, VDW_BMH = 3, VDW_BUFF = 4, VDW_SAAP = 5 };

// surface-correction reduction: blocks of partial sums and sums per block
constexpr int CG_SCAL = 8;     // iterations, final RMS change, ...
constexpr int CG_TRACE = 64;   // RMS change of each iteration of the last solve
constexpr int SURF_BLOCKS = 64, SURF_SUMS = 11;

// Per type pair parameters of the short-range pair term (ntypes^2 rows of 8).
//   LJ : p0 sigma^2, p1 4 eps, p2 energy at the cutoff (shift), p3 unused
//   MIE: p0 sigma, p1 Cn*eps, p2 n, p3 m
//   BMH: p0 A, p1 1/rho, p2 C, p3 D
struct CellGrid {
    int use_cells;
    int n[3];
    int ncell;
    double len[3], rlen[3], origin[3];
    double L0[3];       // the box the grid was laid out for (the barostat scales it)
};

struct PairList {
    int max_nbr = 0;
    int *nbr = nullptr;      // [max_nbr][N]; bit 31 set = same molecule
    int *nnbr = nullptr;     // [N]
    int *cell_of = nullptr, *cell_slot = nullptr, *cell_count = nullptr;
    int *cell_start = nullptr, *cell_atoms = nullptr;
    int cell_cap = 0;
    double rl2 = 0;          // (cutoff + cutBuff)^2
    double drmax = 0;        // cutBuff^2 / 4
};

struct Recip {               // Ewald reciprocal space (k half-space, k^2 < kcut^2)
    int nk = 0;
    int *kn = nullptr;       // [3][nk] integer lattice indices
    double *kcoef = nullptr; // [nk] 4 pi/V * exp(-k^2/4a^2)/k^2
    long long *sk = nullptr; // [2][nk] structure factor, fixed point (SK_SCALE)
    double *kvec = nullptr;  // [3][nk] k in 1/nm
    int nmax = 0;            // largest |n| of any component
    // sheared cell (SLLOD, point charges): the k list depends on the
    // Lees-Edwards offset, so it is rebuilt on the device before every
    // evaluation; nk is then the candidate capacity and nk_dev the count
    int le = 0;
    int le_nx = 0, le_ny = 0, le_nz = 0;   // candidates nx 0..le_nx, ny - round(nx t) and nz within +-le_ny, +-le_nz
    int *nk_dev = nullptr;
    // FP32 passes of the polarisable model (built once per k set; the k list
    // is ordered column by column, nz ascending by one within a column)
    int nseg = 0, ncol = 0, ngrp = 0, row = 0, tab_n = 0;
    int4 *kseg = nullptr;    // sums pass: runs of <= 4 k of one column (first k, count, nx | ny << 16, first nz)
    int4 *kcol = nullptr;    // force pass: columns (first k, length, nx | ny << 16, first nz)
    int4 *kgrp = nullptr;    // force pass: groups of whole columns (first column, columns, first k, k count)
    float4 *kzr = nullptr;   // per k (kz, kz^2, 2c, 0)
    float2 *kcxy = nullptr;  // per column (kx, ky)
    float2 *stab = nullptr;  // per site phase tables [n][row]: e^{2 pi i m f / 2^32}, m < nmax + 1, per axis
    // the FP64 column passes: (kz, kz^2, 2c, 0) per k, (kx, ky) per column,
    // phase tables e^{2 pi i m f / 2^64} and FP64 site records [n][4]
    double4 *kzr_d = nullptr;
    double2 *kcxy_d = nullptr;
    double2 *stab_d = nullptr;
    double4 *srec_d = nullptr;
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    // sizes
    int n = 0, nmol = 0, ntypes = 0;
    // host topology
    std::vector<int> h_type, h_mol, h_mol_off, h_mol_atoms, h_excl_off, h_excl;
    std::vector<double> h_mass, h_charge;
    std::vector<double> h_type_charge;
    double total_mass = 0;
    // device topology
    int *type = nullptr, *mol = nullptr, *mol_off = nullptr, *mol_atoms = nullptr;
    int *excl_off = nullptr, *excl = nullptr;
    double *mass = nullptr;
    double *pair_par = nullptr;    // [ntypes*ntypes*4]
    float *pair_par_f = nullptr;
    double *type_q = nullptr;      // scaled charge per type
    // state
    double4 *pos4 = nullptr, *vel4 = nullptr, *vtm4 = nullptr, *disp4 = nullptr;
    int4 *fixq = nullptr;
    long long *frc = nullptr;      // [3][N]
    long long *acc = nullptr;      // [ACC_COUNT]
    double *scal = nullptr;        // integrator scalars (see smd_integrate.cu)
    double *partials = nullptr;    // per-block reduction partials
    unsigned int *ticket = nullptr;
    unsigned int *status = nullptr;
    int *flags = nullptr;          // [0] rebuild list, [1] list builds so far
    smd_observables *obs = nullptr;  // observables of the last step, on device
    double *series = nullptr;      // recorded per-step samples
    int series_cap = 0;
    // configuration
    Box box{};
    CellGrid grid{};
    PairList pl;
    Recip rc;
    int precision = SMD_PREC_FP64;
    int reference_forms = 0;        // FP64 path: pow() buffered 14-7 and one sine/cosine per (site, k) reciprocal sums
    int want_cells = 1;
    // polarisable multipole model (Multipole / Induction / BuffvdWForce)
    int mp_on = 0, ind_on = 0;
    double mp_rc2 = 0;              // real-space cutoff^2 (cutoffEw)
    double ind_cut2 = 0;            // cutoffInd^2
    double thole_a = 0.39;
    int ind_amoeba = 0;              // induced real space: 0 Thole-damped B_n, 1 Tinker's AMOEBA form
    double *type_mp = nullptr;      // [ntypes][9] local dipole (3) + quadrupole (6)
    double *type_polar = nullptr;   // [ntypes] polarisabilities (nm^3)
    std::vector<double> h_type_polar;
    double *mu = nullptr;           // [3][N] lab-frame dipoles (e nm)
    double *qd = nullptr;           // [6][N] lab-frame quadrupoles (already /3)
    long long *trq = nullptr;       // [3][N] torques, fixed point
    double *e0 = nullptr;           // [3][N] permanent field at the sites
    double *pind = nullptr;         // [3][N] induced dipoles
    float4 *srec = nullptr;         // [N][4] mixed path, FP32: (q, mu), (Qxx, Qxy, Qxz, Qyy), (Qyz, Qzz, px, py), (pz, 0, 0, 0)
    double *cgw = nullptr;          // CG work: r, w, p [3][N] each, alpha [N], two gather copies [N][4], s, u [3][N]
    double *cgs = nullptr;          // CG scalars [CG_SCAL], trace [CG_TRACE], partials [4][blocks][4]
    int cg_max_iter = 500;
    double cg_tol = 2.0819e-8;      // RMS dipole change tolerance (e nm); 1e-6 D
    int cg_guess = 0;               // SMD_GUESS_*: 0 block solution of E0, 1 previous step, 2 learned, 3 first order
    int cg_blocks = 0;
    int pp_blocks = 0;              // grid of the pipelined solve (0: the layout does not allow it)
    int cg_pipelined = 1;           // pipelined solve (molecule blocks): 0 never, 1 mixed path, 2 both precisions
    int cg_precond = SMD_PRECOND_MOLECULE;  // dipole-solve preconditioner
    double *cg_blk = nullptr;       // [nmol][81] inverse molecule blocks of A
    unsigned int *cg_bar = nullptr; // grid barrier: [0] counter, [1] abort word of the launch
    unsigned long long wait_ns = 1000000000ull;  // limit of one device-side barrier wait (1 s)
    int test_skip_block = -1;       // failure-path test: solve block that never arrives
    int *ind_rj = nullptr;          // damped-tensor rows of the solve: partners [N][cap]
    void *ind_rc = nullptr;         // coefficients [N][cap] (float4 or double4)
    int *ind_cnt = nullptr;         // row lengths [N]
    int ind_cap = 0;
    double *phist = nullptr;        // last 4 steps' converged dipoles and fields [4][6][N] (ring, count in flags[2])
    int in_step = 0;                // enqueueing the step graph: the solve stores its dipoles
    double *frame = nullptr;        // [9][N] site axes u, v, w (lab frame)
    // per-site network giving the initial induced dipoles (smd_mlp.cu)
    int mlp_ready = 0;
    int mlp_base = 2;                // order of the extrapolated guess the network corrects
    int mlp_tc = 1;                  // inference and evaluation: 1 tcgen05 tiles of 128 rows, 0 warp-level mma.sync
    float *mlp_w = nullptr;         // parameters, MLP_NPARAM floats
    float *mlp_m = nullptr, *mlp_v = nullptr;  // Adam moments
    float *mlp_part = nullptr;      // per-block gradient partials
    float *mlp_norm = nullptr;      // feature mean [F] and 1/std [F]
    float *mlp_x = nullptr;         // [N][F] raw features of the current configuration
    float *mlp_data = nullptr;      // training rows [cap][F + 3]
    long long mlp_rows = 0, mlp_cap = 0;
    int mlp_t = 0;                  // Adam step count
    // buffered 14-7 with virtual H sites
    int buff_on = 0;
    double buff_n = 14, buff_m = 7, buff_delta = 0.07, buff_gamma = 0.12, buff_h = 0.91;
    double buff_c[6] = {0, 0, 0, 0, 0, 0};
    double buff_sw = 0;             // taper start (nm)
    double4 *vpos4 = nullptr;       // virtual site positions
    int4 *vfixq = nullptr;          // their 32-bit box fractions
    long long *fv = nullptr;        // [3][N] forces on the virtual sites
    int has_multisite = 0;          // some molecule has more than one site
    // bonded terms of flexible molecules (smd_bonded.cu)
    int nbond = 0, nangle = 0, bond_form = 1, ub_on = 0;
    double ub_k = 0, ub_l0 = 0;
    int4 *bonds = nullptr;          // (atom1, atom2, type, 0)
    int4 *angles = nullptr;         // (atom1, atom2, atom3, type)
    double2 *bond_par = nullptr;    // per type (r0, k)
    double2 *angle_par = nullptr;   // per type (theta0, k)
    // radial distribution function (smd_rdf.cu)
    int rdf_nbins = 0;
    long long rdf_samples = 0;
    double rdf_maxr = 0;
    unsigned long long *rdf_hist = nullptr;  // [ntypes][ntypes][nbins]
    int excl_intermol = 0;          // some exclusion joins two molecules
    // Atom::realPos bookkeeping: box shifts per molecule since the last
    // position upload, and the uploaded offsets realPos - position
    double *wrap = nullptr;         // [3][nmol]
    std::vector<double> h_real_off; // [3N] (empty: realPos = position at upload)
    // running averages of the step observables (smd_integrate.cu)
    double *avg = nullptr;          // [AVG_COUNT] sums, updated by every step
    // surface-dipole corrections (smd_surface.cu)
    int surface_on = 0;
    double *surf_part = nullptr;    // per-block partial sums
    double *surf_tot = nullptr;     // the sums
    double *clen2 = nullptr;        // [nmol][3] squared SHAKE distances
    int fixq_from_integrate = 0;    // step graph: integrate writes fixq
    int vdw = VDW_NONE;
    double cutoff = 1.0, cut_buffer = 0.1;
    double vdw_rc2 = 1.0, sw_rs2 = 0.0, sw_c1 = 0, sw_c2 = 0, sw_c3 = 0;
    int switch_on = 0;
    double e_lrc = 0, v_lrc = 0;
    double *saap = nullptr;         // SAAP pair parameters a0..a5 per type pair
    // Wolf summation of the charges (WolfForce)
    int wolf_on = 0;
    double wolf_alpha = 0, wolf_rc = 0, wolf_d = 0;
    int wolf_msites = 0;            // some charge sits on a displaced site
    int *wolf_msite = nullptr;      // per site: 1 if its charge is displaced
    double4 *wpos4 = nullptr;       // charge-site positions
    // isotropic barostat of the chain integrator (NHIntegrator's NpT run)
    int npt = 0;
    double npt_press = 0;           // target pressure, kJ/mol/nm^3
    double npt_tau = 0;             // BarosConst (ps)
    double npt_lrc_k = 0;           // tail-correction energy x volume
    double npt_smin = 0;            // smallest box scale the cell grid covers
    Box *dbox = nullptr;            // the box on the device while the barostat runs
    int ewald_on = 0;
    double ew_alpha = 0, ew_kcut = 0, ew_rc2 = 0, e_self = 0;
    int long_steps = 1;
    smd_integrator_params ip{};
    int integrator_ready = 0;
    int tpp = 8;                    // threads per site in the pair kernel
    int nb_blocks = 0;              // blocks of the integrate kernel
    long long steps_done = 0;
    int list_valid = 0;
    int list_built = 0;      // a pair list exists for the current set-up (its sites may have moved within the skin)
    double4 *upload4 = nullptr;  // staging of uploaded positions
    double *fout = nullptr;      // [3N] device force output of smd_compute_forces, allocated once
    // configuration version: bumped by every call that moves the sites or
    // changes the model or the solver; smd_compute_forces solves the induced
    // dipoles only when they were not solved for the current version
    long long cfg_version = 1;
    long long dip_version = 0;
    // scratch of the on-demand volume derivatives (smd_lustig.cu)
    double4 *lus_com = nullptr;     // [nmol] molecular centres of mass
    double *lus_buf = nullptr;      // per-block / per-k partial sums
    size_t lus_cap = 0;
    // CUDA graph of one step
    cudaGraphExec_t step_graph = nullptr;
    int graph_dirty = 1;
};

// launchers (each enqueues on ctx.stream)
void launch_fixq(Ctx &c);
void launch_upload_positions(Ctx &c);
void launch_nlist(Ctx &c, bool force_rebuild);
void launch_pair(Ctx &c);
void launch_recip(Ctx &c);
void launch_integrate(Ctx &c);
void launch_start_velocities(Ctx &c);
void launch_nhc_first(Ctx &c);
void launch_nhc_second(Ctx &c);
void launch_nhc_start(Ctx &c);
void launch_finalize_forces(Ctx &c, double *f_out_dev);
void launch_intra(Ctx &c);
// polarisable model: term groups (each maps its own torques to forces)
void launch_mp_short(Ctx &c);
void launch_mp_long(Ctx &c);
void launch_ind_solve(Ctx &c);
void launch_ind_field(Ctx &c);
void launch_ind_cg(Ctx &c);
void launch_ind_short(Ctx &c);
void launch_mp_mol(Ctx &c);
bool polar_short_fused(const Ctx &c);
void launch_polar_short(Ctx &c);
inline void touch(Ctx &c) { c.cfg_version++; }
void launch_ind_long(Ctx &c);
void launch_polar_long(Ctx &c);
void launch_torques_end(Ctx &c);
void launch_frames(Ctx &c);
void launch_bonded(Ctx &c, bool bond, bool angle, bool ub);
void launch_intra_flex(Ctx &c, bool mp, bool ind);
int rdf_sample(Ctx &c);
void launch_surface(Ctx &c, bool ewald, bool mp, bool ind);
inline bool has_bonded(const Ctx &c) { return c.nbond > 0 || c.nangle > 0 || c.ub_on; }

// Running sums of the step observables (the energy and stress averages of
// Ensemble::accumulate, src/Ensemble.cpp:814-894), added by the last block
// of every step, in the layout of smd_averages after its sample count:
// [0] samples, [1..11] energies, [12..21] atomic and molecular stress,
// [22..39] atomic and molecular pressure tensors.
constexpr int AVG_COUNT = 40;
__device__ __forceinline__ void accumulate_averages(double *s, const smd_observables &o) {
    if (!s) return;
    const double et = o.e_potential + o.ke_atom;
    s[0] += 1.0;
    s[1] += o.e_potential; s[2] += o.e_potential * o.e_potential;
    s[3] += et; s[4] += et * et;
    s[5] += o.ke_atom; s[6] += o.ke_atom * o.ke_atom;
    s[7] += o.ke_mol; s[8] += o.ke_mol * o.ke_mol;
    s[9] += o.ke_mol != 0.0 ? 1.0 / o.ke_mol : 0.0;
    s[10] += o.volume; s[11] += o.volume * o.volume;
    const double *P[2] = {o.atom_pressure, o.mol_pressure};
    for (int t = 0; t < 2; t++) {
        const double *p = P[t];
        double *d = s + 12 + 5 * t;
        d[0] += (p[0] + p[4] + p[8]) / 3.0;
        d[1] += (p[1] + p[3]) * 0.5;   // shear stress (XY + YX) / 2
        d[2] += (p[3] - p[1]) * 0.5;   // antisymmetric part (YX - XY) / 2
        d[3] += p[0] - p[4];           // first normal stress difference
        d[4] += p[4] - p[8];           // second normal stress difference
        for (int q = 0; q < 9; q++) s[22 + 9 * t + q] += p[q];
    }
}

// the energy components of the accumulator slots (energy[SMD_E_COUNT]);
// e_lrc and e_self are the constant tail and self energies added to the
// vdW and self slots
__host__ __device__ inline void acc_energies(const long long *acc, double e_lrc, double e_self, double *en) {
    for (int q = 0; q < SMD_E_COUNT; q++) en[q] = 0.0;
    en[SMD_E_VDW] = (double)acc[ACC_E_VDW] * ACC_INV + e_lrc;
    en[SMD_E_REAL] = (double)acc[ACC_E_REAL] * ACC_INV;
    en[SMD_E_LONG] = (double)acc[ACC_E_LONG] * ACC_INV;
    en[SMD_E_CORRECT] = e_self + (double)acc[ACC_E_SELF] * ACC_INV;
    en[SMD_E_MOLCORRECT] = (double)acc[ACC_E_INTRA] * ACC_INV;
    en[SMD_E_SURF] = (double)acc[ACC_E_SURF] * ACC_INV;
    en[SMD_E_POL_REAL] = (double)acc[ACC_E_POL_REAL] * ACC_INV;
    en[SMD_E_POL_LONG] = (double)acc[ACC_E_POL_LONG] * ACC_INV;
    en[SMD_E_POL_SELF] = (double)acc[ACC_E_POL_SELF] * ACC_INV;
    en[SMD_E_POL_INTRA] = (double)acc[ACC_E_POL_INTRA] * ACC_INV;
    en[SMD_E_POL_SURF] = (double)acc[ACC_E_POL_SURF] * ACC_INV;
    en[SMD_E_BOND] = (double)acc[ACC_E_BOND] * ACC_INV;
    en[SMD_E_ANGLE] = (double)acc[ACC_E_ANGLE] * ACC_INV;
    en[SMD_E_UB] = (double)acc[ACC_E_UB] * ACC_INV;
}
void launch_buff(Ctx &c);
int setup_cg(Ctx &c);
int recip_nk(Ctx &c, int *nk);
int ensure_ind_rows(Ctx &c);
// dipole-guess network (smd_mlp.cu)
int mlp_alloc(Ctx &c, long long cap_rows, unsigned int seed);
void launch_mlp_guess(Ctx &c);
void launch_first_order_guess(Ctx &c);
void launch_blk_response(Ctx &c, double *out, int order, double *out_prev);
int lustig_lj(Ctx &c, double *out);
int lustig_all(Ctx &c, double *out);
void launch_wolf_sites(Ctx &c);
void launch_mp_real_only(Ctx &c);
void launch_ind_real_only(Ctx &c);
void launch_ind_self_only(Ctx &c);
void launch_intra_flex_lus(Ctx &c, bool mp, bool ind, double *fr_mol);
// order of the extrapolated guess of the solver's guess mode (0: none)
inline int guess_order(const Ctx &c) {
    return c.cg_guess == SMD_GUESS_FIRST_ORDER ? 1
           : c.cg_guess == SMD_GUESS_EXTRAP2   ? 2
           : c.cg_guess == SMD_GUESS_EXTRAP3   ? 3
                                               : 0;
}
// first-order part of the learned guess: the solver's s slot of its work
// area, which the solve writes before it first reads it
inline double *guess_response(Ctx &c) { return c.cgw + 20 * (size_t)c.n; }
// M^-1 (E0(t-1) - E0(t-2)), the network's input (the solve's residual
// buffer, free until the solve starts)
inline double *guess_response_prev(Ctx &c) { return c.cgw; }
int mlp_batch_loss(Ctx &c, const unsigned int *perm, int batch, double *loss);
void launch_mlp_features(Ctx &c);
void launch_mlp_collect(Ctx &c);
void launch_mlp_norm(Ctx &c);
void launch_mlp_step(Ctx &c, const unsigned int *perm, long long r0, int batch, float lr, float *grad_out);
void launch_mlp_eval(Ctx &c, int rows, const float *x, float *y);
int mlp_nparam();
int mlp_nfeat();
int mlp_max_batch();
int setup_recip(Ctx &c);
int mp_recip_prepare(Ctx &c);

}  // namespace smd
