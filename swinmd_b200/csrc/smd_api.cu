// C-ABI entry points (declared in include/swinmd_b200.h): context lifetime,
// topology and parameter upload, force evaluation and the integration loop.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <new>
#include <string>
#include "smd_ctx.cuh"

using namespace smd;

struct smd_ctx {
    Ctx c;
};

// ---- scratch of the force evaluation without device allocation ------------
// The device output buffer of smd_compute_forces_noalloc lives in this
// file-scope array instead of the context's buffer.  Nothing in it needs to
// start at zero: the finalize kernel writes every element a call reads back.
// One array per process and device: calls that overlap (two threads, or two
// contexts on one device) share it and race.
namespace {
constexpr int NOALLOC_MAX_SITES = 65536;
static __device__ __align__(256) double g_noalloc_force[3 * NOALLOC_MAX_SITES];
constexpr int NOALLOC_MAX_DEVICES = 64;
// the array's device address per device, resolved once with that device
// current; cleared when the last context of the device is destroyed, so a
// device reset followed by new contexts resolves it again
std::mutex g_noalloc_mu;
double *g_noalloc_addr[NOALLOC_MAX_DEVICES] = {nullptr};
int g_live_ctx[NOALLOC_MAX_DEVICES] = {0};
}  // namespace

namespace {

int fail(smd_ctx *x, int code, const std::string &msg) {
    if (x) x->c.err = msg;
    return code;
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(x, SMD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
cudaError_t dalloc(T **p, size_t count) {
    if (*p) cudaFree(*p);
    *p = nullptr;
    if (count == 0) count = 1;
    return cudaMalloc((void **)p, count * sizeof(T));
}

int status_to_code(unsigned st) {
    if (st & ST_BOX) return SMD_ERR_BOX;   // first: what follows it may stem from it
    if (st & ST_LIST_OVERFLOW) return SMD_ERR_LIST_OVERFLOW;
    if (st & ST_NAN) return SMD_ERR_NAN;
    if (st & (ST_SHAKE_ITER | ST_SHAKE_GEOM)) return SMD_ERR_SHAKE;
    if (st & ST_NH_ITER) return SMD_ERR_NH_ITER;
    if (st & ST_WAIT_TIMEOUT) return SMD_ERR_TIMEOUT;
    if (st & ST_CG_ITER) return SMD_ERR_CG;
    return SMD_OK;
}

const char *status_text(unsigned st) {
    if (st & ST_BOX) return "the barostat shrank the box below the cell grid's reach";
    if (st & ST_LIST_OVERFLOW) return "pair list overflow: a site has more neighbours than the list holds";
    if (st & ST_NAN) return "non-finite position";
    if (st & ST_SHAKE_GEOM) return "SHAKE geometric failure";
    if (st & ST_SHAKE_ITER) return "SHAKE did not converge within maxCount";
    if (st & ST_NH_ITER) return "NH iteration Error";
    if (st & ST_WAIT_TIMEOUT)
        return "dipole solve: a grid-barrier wait ran out (solve blocks not all resident, or one never arrived)";
    if (st & ST_CG_ITER) return "dipole solve did not converge";
    return "";
}

// Cell grid as CellManager::set_cellManager (src/utils/CellManager.cpp:43-84).
void setup_grid(Ctx &c, int use_cells) {
    CellGrid &g = c.grid;
    double len = c.cutoff + c.cut_buffer;
    g.use_cells = use_cells;
    for (int d = 0; d < 3; d++) g.L0[d] = c.box.L[d];
    // with the barostat the cells are laid out for a box 10 % smaller, so
    // that the 27-cell stencil still covers the list radius as it shrinks
    const double room = c.npt ? 0.9 : 1.0;
    for (int d = 0; d < 3; d++)
        if (len <= 0 || len > room * c.box.L[d] / 3.0) g.use_cells = 0;
    if (!g.use_cells) {
        g.ncell = 0;
        for (int d = 0; d < 3; d++) { g.n[d] = 0; g.len[d] = g.rlen[d] = g.origin[d] = 0; }
        return;
    }
    for (int d = 0; d < 3; d++) {
        g.n[d] = (int)(room * c.box.L[d] / len);
        g.len[d] = c.box.L[d] / g.n[d];
        g.rlen[d] = 1.0 / g.len[d];
        g.origin[d] = -c.box.L[d] / 2.0;
    }
    g.ncell = g.n[0] * g.n[1] * g.n[2];
}

int alloc_list(smd_ctx *x) {
    Ctx &c = x->c;
    if (c.n == 0 || c.box.L[0] <= 0) return SMD_OK;
    double rl = c.cutoff + c.cut_buffer;
    double vol = c.box.L[0] * c.box.L[1] * c.box.L[2];
    double dens = c.n / vol;
    double expect = 4.18879020478639 * rl * rl * rl * dens;
    int cap = (int)(expect * 1.6 + 64);
    cap = (cap + 31) & ~31;
    cap = std::min(cap, c.n);
    cap = std::max(cap, 32);
    if (cap != c.pl.max_nbr || !c.pl.nbr) {
        c.pl.max_nbr = cap;
        CK(dalloc(&c.pl.nbr, (size_t)cap * c.n));
    }
    int ncell = std::max(c.grid.ncell, 1);
    if (ncell > c.pl.cell_cap) {
        CK(dalloc(&c.pl.cell_count, ncell));
        CK(dalloc(&c.pl.cell_start, ncell + 1));
        CK(cudaMemset(c.pl.cell_count, 0, ncell * sizeof(int)));
        c.pl.cell_cap = ncell;
    }
    c.list_valid = 0;
    c.list_built = 0;
    c.graph_dirty = 1;
    touch(c);
    if (ensure_ind_rows(c)) return fail(x, SMD_ERR_CUDA, "dipole-solve tensor rows: allocation failed");
    return SMD_OK;
}

int sync_status(smd_ctx *x) {
    Ctx &c = x->c;
    CK(cudaStreamSynchronize(c.stream));
    CK(cudaGetLastError());
    unsigned st = 0;
    CK(cudaMemcpy(&st, c.status, sizeof(unsigned), cudaMemcpyDeviceToHost));
    int code = status_to_code(st);
    if (code != SMD_OK) return fail(x, code, status_text(st));
    return SMD_OK;
}

// Polarisable model, in the order LFIntegrator::run calls the reference's
// terms (LFIntegrator.cpp:440-458): multipoles short and long, then the
// induced dipoles (solved once per step) short and long; all torques are
// mapped onto the sites at the end (the mapping is linear in the torques).
// solved: the induced dipoles (and the solve's tensor rows) already belong
// to the current configuration, as after an earlier smd_compute_forces on
// it; the reference's Induction::compute_long likewise uses the dipoles its
// compute() solved (src/forces/Induction.cpp:567-590).
void enqueue_polar(Ctx &c, bool mp_short, bool mp_long, bool ind_short, bool ind_long, bool solved = false) {
    launch_frames(c);   // also the site records (with the current dipoles) and cleared torques
    const bool all = mp_short && mp_long && ind_short && ind_long && c.ind_on;
    if (all && polar_short_fused(c)) {
        // mixed path: the multipole real space does not feed the solve, so
        // it runs after it, fused with the induced real space
        if (!solved) launch_ind_solve(c);
        launch_polar_short(c);
        launch_polar_long(c);
        launch_surface(c, false, true, true);
        launch_torques_end(c);
        return;
    }
    if (mp_short) launch_mp_short(c);
    if (all) {
        // a full evaluation: after the solve one pass gives all structure
        // factors and one reciprocal force pass serves both terms
        if (!solved) launch_ind_solve(c);
        launch_ind_short(c);
        launch_polar_long(c);
    } else {
        if (mp_long) launch_mp_long(c);
        if (c.ind_on && (ind_short || ind_long)) {
            if (!solved) launch_ind_solve(c);
            if (ind_short) launch_ind_short(c);
            if (ind_long) launch_ind_long(c);
        }
    }
    // Multipole::compute and Induction::compute add their surface terms
    launch_surface(c, false, mp_short, ind_short && c.ind_on);
    launch_torques_end(c);
}

void enqueue_forces(Ctx &c) {
    launch_pair(c);
    if (c.ewald_on) {
        launch_intra(c);
        launch_recip(c);
        launch_surface(c, true, false, false);
    }
    if (c.mp_on) enqueue_polar(c, true, true, true, true);
    if (has_bonded(c)) launch_bonded(c, true, true, true);
}

// One MD step: in the FP32 path the integrate kernel of the previous step
// (or smd_integrator_start / smd_upload_positions) has already written the
// box fractions the pair kernel reads.
void enqueue_step(Ctx &c) {
    if (c.ip.thermostat == SMD_THERMO_NH_CHAIN) {
        // velocity Verlet: chain, kick and drift first, then the list test,
        // forces at t + dt, the second kick and chain
        launch_nhc_first(c);
        launch_nlist(c, false);
        c.fixq_from_integrate = 1;
        c.in_step = 1;
        enqueue_forces(c);
        c.in_step = 0;
        c.fixq_from_integrate = 0;
        launch_nhc_second(c);
        return;
    }
    launch_nlist(c, false);
    c.fixq_from_integrate = 1;
    c.in_step = 1;
    enqueue_forces(c);
    c.in_step = 0;
    c.fixq_from_integrate = 0;
    launch_integrate(c);
}


// One evaluation of the selected terms at the current positions into the
// device buffer dforce (3N doubles, used only when force is given), then the
// forces, energies and virial copied to the host.  The pair list is kept
// while every site stays within half the skin of its last build (the test a
// step makes); the induced dipoles are solved once per configuration.
int compute_forces_into(smd_ctx *x, uint32_t terms, double *dforce, double *force, double *energy,
                        double *virial) {
    Ctx &c = x->c;
    CK(cudaMemsetAsync(c.status, 0, sizeof(unsigned), c.stream));
    const bool rebuild = !c.list_built;
    launch_nlist(c, rebuild);
    // smd_get_pairs returns the list of the current positions: a kept list
    // (built at earlier positions) is rebuilt there first
    c.list_valid = rebuild ? 1 : 0;
    CK(cudaMemsetAsync(c.acc, 0, ACC_COUNT * sizeof(long long), c.stream));
    CK(cudaMemsetAsync(c.frc, 0, 3 * (size_t)c.n * sizeof(long long), c.stream));
    const int save_vdw = c.vdw, save_ew = c.ewald_on, save_wolf = c.wolf_on;
    if (!(terms & SMD_TERM_VDW)) c.vdw = VDW_NONE;
    if (!(terms & SMD_TERM_WOLF)) c.wolf_on = 0;
    bool want_real = (terms & SMD_TERM_EWALD_REAL) && c.ewald_on;
    bool want_long = (terms & SMD_TERM_EWALD_LONG) && c.ewald_on;
    c.ewald_on = want_real ? 1 : 0;
    launch_pair(c);
    if (want_real) {
        launch_intra(c);
        launch_surface(c, true, false, false);   // EwaldForce::compute adds its surface term
    }
    c.ewald_on = save_ew;
    c.wolf_on = save_wolf;
    if (want_long) launch_recip(c);
    c.vdw = save_vdw;
    if (has_bonded(c))
        launch_bonded(c, terms & SMD_TERM_BOND, terms & SMD_TERM_ANGLE, terms & SMD_TERM_UB);
    const uint32_t polar = SMD_TERM_MP_SHORT | SMD_TERM_MP_LONG | SMD_TERM_IND_SHORT | SMD_TERM_IND_LONG;
    if (c.mp_on && (terms & polar)) {
        const bool solved = c.ind_on && c.dip_version == c.cfg_version;
        enqueue_polar(c, terms & SMD_TERM_MP_SHORT, terms & SMD_TERM_MP_LONG, terms & SMD_TERM_IND_SHORT,
                      terms & SMD_TERM_IND_LONG, solved);
    }
    if (force) launch_finalize_forces(c, dforce);
    long long hacc[ACC_COUNT];
    CK(cudaMemcpyAsync(hacc, c.acc, sizeof(hacc), cudaMemcpyDeviceToHost, c.stream));
    // a time step starts from cleared accumulators (the integrator clears
    // them at the end of every step): leave them so for the next smd_run
    CK(cudaMemsetAsync(c.acc, 0, ACC_COUNT * sizeof(long long), c.stream));
    if (force) CK(cudaMemcpyAsync(force, dforce, 3 * (size_t)c.n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    const int rs = sync_status(x);
    if (rs) {
        c.dip_version = 0;   // a failed evaluation leaves no usable dipoles
        return rs;
    }
    if (c.mp_on && c.ind_on && (terms & (SMD_TERM_IND_SHORT | SMD_TERM_IND_LONG)))
        c.dip_version = c.cfg_version;   // solved now, or already before
    const bool vdw = (terms & SMD_TERM_VDW) && c.vdw != VDW_NONE;
    if (energy) acc_energies(hacc, vdw ? c.e_lrc : 0.0, want_real ? c.e_self : 0.0, energy);
    if (virial) {
        for (int q = 0; q < 9; q++) {
            virial[q] = ((double)hacc[ACC_VIR + q] + (double)hacc[ACC_LVIR + q]) * ACC_INV;
            if (vdw && (q == 0 || q == 4 || q == 8)) virial[q] -= c.v_lrc;
        }
    }
    return SMD_OK;
}
}  // namespace

extern "C" {

int smd_create(int device, smd_ctx **out) {
    smd_ctx *x = nullptr;
    if (!out) return SMD_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return SMD_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return SMD_ERR_ARG;
    x = new (std::nothrow) smd_ctx();
    if (!x) return SMD_ERR_ARG;
    Ctx &c = x->c;
    c.device = device;
    if (cudaSetDevice(device) != cudaSuccess) { delete x; return SMD_ERR_CUDA; }
    if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete x;
        return SMD_ERR_CUDA;
    }
    if (dalloc(&c.acc, ACC_COUNT) != cudaSuccess || dalloc(&c.scal, SC_NSCAL) != cudaSuccess ||
        dalloc(&c.ticket, 1) != cudaSuccess || dalloc(&c.status, 1) != cudaSuccess ||
        dalloc(&c.flags, 4) != cudaSuccess || dalloc(&c.obs, 1) != cudaSuccess ||
        dalloc(&c.avg, AVG_COUNT) != cudaSuccess) {
        delete x;
        return SMD_ERR_CUDA;
    }
    cudaMemset(c.acc, 0, ACC_COUNT * sizeof(long long));
    cudaMemset(c.scal, 0, SC_NSCAL * sizeof(double));
    cudaMemset(c.ticket, 0, sizeof(unsigned));
    cudaMemset(c.status, 0, sizeof(unsigned));
    cudaMemset(c.flags, 0, 4 * sizeof(int));
    cudaMemset(c.obs, 0, sizeof(smd_observables));
    cudaMemset(c.avg, 0, AVG_COUNT * sizeof(double));
    if (device < NOALLOC_MAX_DEVICES) {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        g_live_ctx[device]++;
    }
    *out = x;
    return SMD_OK;
}

void smd_destroy(smd_ctx *x) {
    if (!x) return;
    Ctx &c = x->c;
    cudaSetDevice(c.device);
    if (c.step_graph) cudaGraphExecDestroy(c.step_graph);
    void *ptrs[] = {c.type, c.mol, c.mol_off, c.mol_atoms, c.excl_off, c.excl, c.mass,
                    c.pair_par, c.pair_par_f, c.type_q, c.pos4, c.vel4, c.vtm4, c.disp4, c.fixq,
                    c.frc, c.acc, c.scal, c.partials, c.ticket, c.status, c.flags, c.obs,
                    c.series, c.pl.nbr, c.pl.nnbr, c.pl.cell_of, c.pl.cell_slot,
                    c.pl.cell_count, c.pl.cell_start, c.pl.cell_atoms, c.rc.kn, c.rc.kcoef,
                    c.rc.sk, c.rc.kvec, c.clen2, c.type_mp, c.type_polar, c.mu, c.qd, c.trq, c.e0,
                    c.pind, c.cgw, c.cgs, c.cg_bar, c.vpos4, c.vfixq, c.fv, c.ind_rj, c.ind_rc, c.ind_cnt,
                    c.rc.kseg, c.rc.kcol, c.rc.kgrp, c.rc.kzr, c.rc.kcxy, c.rc.stab, c.srec, c.phist, c.cg_blk,
                    c.upload4, c.fout, c.rc.kzr_d, c.rc.kcxy_d, c.rc.stab_d, c.rc.srec_d, c.bonds, c.angles,
                    c.bond_par, c.angle_par, c.surf_part, c.surf_tot, c.rdf_hist, c.avg, c.wrap,
                    c.wolf_msite, c.wpos4, c.dbox, c.saap, c.rc.nk_dev, c.lus_com, c.lus_buf};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (c.stream) cudaStreamDestroy(c.stream);
    if (c.device >= 0 && c.device < NOALLOC_MAX_DEVICES) {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (--g_live_ctx[c.device] <= 0) {
            g_live_ctx[c.device] = 0;
            g_noalloc_addr[c.device] = nullptr;   // resolved again by the next context's first call
        }
    }
    delete x;
}

const char *smd_last_error(const smd_ctx *x) { return x ? x->c.err.c_str() : "null context"; }

int smd_set_topology(smd_ctx *x, int n, int ntypes, const int32_t *atom_type,
                     const int32_t *mol_id, const double *mass, const double *scaled_charge) {
    if (!x || n <= 0 || ntypes <= 0 || ntypes > 8 || !atom_type || !mol_id || !mass || !scaled_charge)
        return fail(x, SMD_ERR_ARG, "smd_set_topology: bad arguments (ntypes must be 1..8)");
    Ctx &c = x->c;
    CK(cudaSetDevice(c.device));
    c.n = n;
    c.ntypes = ntypes;
    c.h_type.assign(atom_type, atom_type + n);
    c.h_mol.assign(mol_id, mol_id + n);
    c.h_mass.assign(mass, mass + n);
    c.h_charge.assign(scaled_charge, scaled_charge + n);
    int nmol = 0;
    for (int i = 0; i < n; i++) {
        if (atom_type[i] < 0 || atom_type[i] >= ntypes || mol_id[i] < 0)
            return fail(x, SMD_ERR_ARG, "smd_set_topology: atom type or molecule id out of range");
        nmol = std::max(nmol, mol_id[i] + 1);
    }
    c.nmol = nmol;
    // molecule -> atoms in atom order (Molecule::add_atom, src/Ensemble.cpp:216-222)
    c.h_mol_off.assign(nmol + 1, 0);
    for (int i = 0; i < n; i++) c.h_mol_off[mol_id[i] + 1]++;
    for (int m = 0; m < nmol; m++) c.h_mol_off[m + 1] += c.h_mol_off[m];
    c.h_mol_atoms.assign(n, 0);
    std::vector<int> fill(c.h_mol_off.begin(), c.h_mol_off.end() - 1);
    for (int i = 0; i < n; i++) c.h_mol_atoms[fill[mol_id[i]]++] = i;
    for (int m = 0; m < nmol; m++)
        if (c.h_mol_off[m + 1] == c.h_mol_off[m])
            return fail(x, SMD_ERR_ARG, "smd_set_topology: molecule ids must be contiguous from 0");
    // charge per type (Atom::scaledCharge is a per-type parameter)
    c.h_type_charge.assign(ntypes, 0.0);
    std::vector<int> seen(ntypes, 0);
    for (int i = 0; i < n; i++) {
        int t = atom_type[i];
        if (!seen[t]) { c.h_type_charge[t] = scaled_charge[i]; seen[t] = 1; }
        else if (c.h_type_charge[t] != scaled_charge[i])
            return fail(x, SMD_ERR_ARG, "smd_set_topology: charges must be per atom type");
    }
    c.has_multisite = 0;
    for (int m = 0; m < nmol; m++)
        if (c.h_mol_off[m + 1] - c.h_mol_off[m] > 1) c.has_multisite = 1;
    c.total_mass = 0;
    for (int i = 0; i < n; i++) c.total_mass += mass[i];

    CK(dalloc(&c.type, n)); CK(dalloc(&c.mol, n)); CK(dalloc(&c.mass, n));
    CK(dalloc(&c.mol_off, nmol + 1)); CK(dalloc(&c.mol_atoms, n));
    CK(dalloc(&c.type_q, ntypes));
    CK(dalloc(&c.pos4, n)); CK(dalloc(&c.vel4, n)); CK(dalloc(&c.vtm4, n));
    CK(dalloc(&c.disp4, n)); CK(dalloc(&c.fixq, n));
    CK(dalloc(&c.frc, 3 * (size_t)n));
    CK(dalloc(&c.pl.nnbr, n)); CK(dalloc(&c.pl.cell_of, n)); CK(dalloc(&c.pl.cell_slot, n));
    CK(dalloc(&c.pl.cell_atoms, n));
    int nb = (nmol + 31) / 32;   // the integrate kernels' smallest blocks
    CK(dalloc(&c.partials, (size_t)nb * 40));  // per block: NPART (35) partial sums
    CK(dalloc(&c.wrap, 3 * (size_t)nmol));
    CK(cudaMemset(c.wrap, 0, 3 * (size_t)nmol * sizeof(double)));
    c.h_real_off.clear();
    CK(cudaMemcpy(c.type, atom_type, n * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.mol, mol_id, n * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.mass, mass, n * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.mol_off, c.h_mol_off.data(), (nmol + 1) * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.mol_atoms, c.h_mol_atoms.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.type_q, c.h_type_charge.data(), ntypes * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemset(c.disp4, 0, n * sizeof(double4)));
    CK(cudaMemset(c.frc, 0, 3 * (size_t)n * sizeof(long long)));
    // velocity arrays carry 1/m and m in .w
    std::vector<double4> v(n), vm(n);
    for (int i = 0; i < n; i++) {
        v[i] = make_double4(0, 0, 0, 1.0 / mass[i]);
        vm[i] = make_double4(0, 0, 0, mass[i]);
    }
    CK(cudaMemcpy(c.vel4, v.data(), n * sizeof(double4), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.vtm4, vm.data(), n * sizeof(double4), cudaMemcpyHostToDevice));
    // no exclusions until smd_set_exclusions
    std::vector<int> off(n + 1, 0);
    c.h_excl_off = off;
    c.h_excl.clear();
    CK(dalloc(&c.excl_off, n + 1)); CK(dalloc(&c.excl, 1));
    CK(cudaMemcpy(c.excl_off, off.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice));
    // default pair parameters: none
    CK(dalloc(&c.pair_par, (size_t)ntypes * ntypes * 4));
    CK(cudaMemset(c.pair_par, 0, (size_t)ntypes * ntypes * 4 * sizeof(double)));
    c.list_valid = 0;
    c.list_built = 0;
    c.graph_dirty = 1;
    touch(c);
    return alloc_list(x);
}

int smd_set_exclusions(smd_ctx *x, const int32_t *offsets, const int32_t *partners) {
    if (!x || !offsets || x->c.n == 0) return fail(x, SMD_ERR_ARG, "smd_set_exclusions: bad arguments");
    Ctx &c = x->c;
    int n = c.n;
    int tot = offsets[n];
    if (offsets[0] != 0 || tot < 0 || (tot > 0 && !partners))
        return fail(x, SMD_ERR_ARG, "smd_set_exclusions: bad CSR offsets");
    for (int i = 0; i < n; i++)
        if (offsets[i + 1] < offsets[i]) return fail(x, SMD_ERR_ARG, "smd_set_exclusions: offsets decrease");
    for (int k = 0; k < tot; k++)
        if (partners[k] < 0 || partners[k] >= n) return fail(x, SMD_ERR_ARG, "smd_set_exclusions: partner out of range");
    c.h_excl_off.assign(offsets, offsets + n + 1);
    c.h_excl.assign(partners, partners + tot);
    c.excl_intermol = 0;
    for (int i = 0; i < n; i++)
        for (int k = offsets[i]; k < offsets[i + 1]; k++)
            if (c.h_mol[partners[k]] != c.h_mol[i]) c.excl_intermol = 1;
    CK(dalloc(&c.excl, std::max(tot, 1)));
    CK(cudaMemcpy(c.excl_off, offsets, (n + 1) * sizeof(int), cudaMemcpyHostToDevice));
    if (tot) CK(cudaMemcpy(c.excl, partners, tot * sizeof(int), cudaMemcpyHostToDevice));
    c.list_valid = 0;
    c.list_built = 0;
    c.graph_dirty = 1;
    touch(c);
    if (ensure_ind_rows(c)) return fail(x, SMD_ERR_CUDA, "dipole-solve tensor rows: allocation failed");
    return SMD_OK;
}

int smd_set_box(smd_ctx *x, double lx, double ly, double lz) {
    if (!x || !(lx > 0) || !(ly > 0) || !(lz > 0)) return fail(x, SMD_ERR_ARG, "smd_set_box: edges must be > 0");
    Ctx &c = x->c;
    c.box.L[0] = lx; c.box.L[1] = ly; c.box.L[2] = lz;
    for (int d = 0; d < 3; d++) {
        c.box.half[d] = 0.5 * c.box.L[d];
        c.box.inv[d] = 1.0 / c.box.L[d];
    }
    setup_grid(c, c.want_cells);
    if (c.ewald_on || c.mp_on) {
        int r = setup_recip(c);
        if (r) return fail(x, r, "smd_set_box: reciprocal set-up failed");
    }
    if (c.dbox) CK(cudaMemcpy(c.dbox, &c.box, sizeof(Box), cudaMemcpyHostToDevice));
    return alloc_list(x);
}

int smd_lustig_lj(smd_ctx *x, double *out) {
    if (!x || !out || x->c.vdw != VDW_LJ) return fail(x, SMD_ERR_ARG, "smd_lustig_lj: the vdW term is not LJ");
    Ctx &c = x->c;
    CK(cudaSetDevice(c.device));
    int r = lustig_lj(c, out);
    if (r) return fail(x, r, "smd_lustig_lj: evaluation failed");
    return sync_status(x);
}

int smd_lustig(smd_ctx *x, double *out) {
    if (!x || !out || x->c.n == 0 || x->c.box.L[0] <= 0) return fail(x, SMD_ERR_ARG, "smd_lustig: system not set up");
    if (x->c.ind_amoeba && x->c.ind_on)
        return fail(x, SMD_ERR_ARG, "smd_lustig: the AMOEBA-damped induced real space has no volume derivatives here");
    Ctx &c = x->c;
    if (c.rc.le || (c.vdw != VDW_NONE && c.vdw != VDW_LJ && c.vdw != VDW_BUFF))
        return fail(x, SMD_ERR_ARG,
                    "smd_lustig: built for the LJ and buffered 14-7 terms, Ewald and Wolf sums, multipoles, "
                    "induced dipoles and bonded terms (no Mie, BMH, SAAP or sheared cell)");
    CK(cudaSetDevice(c.device));
    CK(cudaMemsetAsync(c.status, 0, sizeof(unsigned), c.stream));
    int r = lustig_all(c, out);
    if (r) return fail(x, r, "smd_lustig: evaluation failed");
    return sync_status(x);
}

int smd_set_saap(smd_ctx *x, const double *table, int switch_on, double switch_dist2) {
    if (!x || !table || x->c.ntypes == 0) return fail(x, SMD_ERR_ARG, "smd_set_saap: set the topology first");
    Ctx &c = x->c;
    const int nt = c.ntypes;
    for (int k = 0; k < 6 * nt * nt; k++)
        if (!std::isfinite(table[k])) return fail(x, SMD_ERR_NAN, "smd_set_saap: non-finite parameter");
    // the switch constants as smd_set_vdw forms them (no parameters of its own)
    int r = smd_set_vdw(x, SMD_VDW_NONE, nullptr, switch_on, switch_dist2, 0.0, 0.0);
    if (r) return r;
    CK(dalloc(&c.saap, (size_t)6 * nt * nt));
    CK(cudaMemcpy(c.saap, table, (size_t)6 * nt * nt * sizeof(double), cudaMemcpyHostToDevice));
    c.vdw = VDW_SAAP;
    // with the switch off the kernel never reads sw_rs2; with it on,
    // smd_set_vdw has set it for a non-LJ kind
    c.graph_dirty = 1;
    touch(c);
    return SMD_OK;
}

int smd_set_wolf(smd_ctx *x, double alpha, double cutoff, const int *msite, double d_op) {
    if (!x || !(alpha > 0) || !(cutoff > 0) || x->c.n == 0 || x->c.ewald_on)
        return fail(x, SMD_ERR_ARG, "smd_set_wolf: set the topology first; alpha, cutoff > 0; not with Ewald");
    Ctx &c = x->c;
    std::vector<int> flag(c.n, 0);
    int any = 0;
    if (msite)
        for (int i = 0; i < c.n; i++) {
            flag[i] = msite[i] ? 1 : 0;
            any |= flag[i];
            if (flag[i] && c.h_mol_off[c.h_mol[i] + 1] - c.h_mol_off[c.h_mol[i]] != 3)
                return fail(x, SMD_ERR_ARG, "smd_set_wolf: a displaced charge site needs a 3-site molecule");
        }
    if (any && !(d_op > 0)) return fail(x, SMD_ERR_ARG, "smd_set_wolf: d_op must be > 0");
    CK(dalloc(&c.wolf_msite, (size_t)c.n));
    CK(cudaMemcpy(c.wolf_msite, flag.data(), c.n * sizeof(int), cudaMemcpyHostToDevice));
    if (any) CK(dalloc(&c.wpos4, (size_t)c.n));
    c.wolf_on = 1;
    c.wolf_alpha = alpha;
    c.wolf_rc = cutoff;
    c.wolf_d = d_op;
    c.wolf_msites = any;
    c.graph_dirty = 1;
    touch(c);
    return SMD_OK;
}

int smd_set_barostat(smd_ctx *x, double pressure, double baros_const, int on) {
    if (!x || (on && !(baros_const > 0)) || !std::isfinite(pressure))
        return fail(x, SMD_ERR_ARG, "smd_set_barostat: BarosConst must be > 0");
    Ctx &c = x->c;
    c.npt = on ? 1 : 0;
    c.npt_press = pressure / 1.66053904042716;   // Integrator.cpp:44
    c.npt_tau = baros_const;
    if (on && !c.dbox) CK(dalloc(&c.dbox, 1));
    if (c.dbox) CK(cudaMemcpy(c.dbox, &c.box, sizeof(Box), cudaMemcpyHostToDevice));
    setup_grid(c, c.want_cells);
    return alloc_list(x);
}

int smd_get_box(smd_ctx *x, double *edges) {
    if (!x || !edges) return SMD_ERR_ARG;
    Ctx &c = x->c;
    Box b = c.box;
    if (c.npt && c.dbox) {
        CK(cudaStreamSynchronize(c.stream));
        CK(cudaMemcpy(&b, c.dbox, sizeof(Box), cudaMemcpyDeviceToHost));
    }
    for (int d = 0; d < 3; d++) edges[d] = b.L[d];
    return SMD_OK;
}

int smd_set_pairlist(smd_ctx *x, double cutoff, double cut_buffer, int use_cells) {
    if (!x || !(cutoff > 0) || cut_buffer < 0) return fail(x, SMD_ERR_ARG, "smd_set_pairlist: bad cutoff");
    Ctx &c = x->c;
    c.cutoff = cutoff;
    c.cut_buffer = cut_buffer;
    double pc = cutoff + cut_buffer;   // Ensemble::set_pairlist, src/Ensemble.cpp:456-457
    pc *= pc;
    c.pl.rl2 = pc;
    c.pl.drmax = cut_buffer * cut_buffer / 4.0;  // Integrator.cpp:36
    c.vdw_rc2 = cutoff * cutoff;
    c.want_cells = use_cells;
    setup_grid(c, use_cells);
    return alloc_list(x);
}

int smd_set_vdw(smd_ctx *x, int kind, const double *params, int switch_on, double switch_dist2,
                double e_lrc, double v_lrc) {
    if (!x || kind < 0 || kind > 3 || (kind != SMD_VDW_NONE && !params) || x->c.ntypes == 0)
        return fail(x, SMD_ERR_ARG, "smd_set_vdw: bad arguments");
    Ctx &c = x->c;
    int nt = c.ntypes;
    std::vector<double> p((size_t)nt * nt * 4, 0.0);
    if (params) std::memcpy(p.data(), params, p.size() * sizeof(double));
    c.vdw = kind;
    c.switch_on = switch_on;
    c.e_lrc = e_lrc;
    c.v_lrc = v_lrc;
    double rc2 = c.vdw_rc2;
    if (kind == SMD_VDW_LJ) {
        // energy at the cutoff (LJForce.cpp:159-166)
        double rcut_2 = 1.0 / rc2;
        for (int k = 0; k < nt * nt; k++) {
            double sr2 = p[4 * k] * rcut_2;
            double sr6 = sr2 * sr2 * sr2;
            double sr12 = sr6 * sr6;
            p[4 * k + 2] = p[4 * k + 1] * (sr12 - sr6);
        }
    }
    // 5th-order switch constants (MieForce.cpp:26-46)
    c.sw_rs2 = rc2;
    if (switch_on) c.sw_rs2 = switch_dist2;
    if (switch_on && rc2 > c.sw_rs2) {
        double c1 = 1.0 / (rc2 - c.sw_rs2);
        c.sw_c1 = c1 * c1 * c1;
        c.sw_c2 = rc2 - 3.0 * c.sw_rs2;
        c.sw_c3 = 4 * c.sw_c1;
    } else {
        c.sw_c1 = c.sw_c2 = c.sw_c3 = 0.0;
        if (kind != SMD_VDW_LJ) c.sw_rs2 = rc2;  // switch inactive
    }
    CK(cudaMemcpy(c.pair_par, p.data(), p.size() * sizeof(double), cudaMemcpyHostToDevice));
    c.graph_dirty = 1;
    touch(c);
    return SMD_OK;
}

int smd_set_ewald(smd_ctx *x, double alpha, double kcut, double real_cut) {
    if (!x || !(alpha > 0) || !(kcut > 0) || !(real_cut > 0) || x->c.n == 0)
        return fail(x, SMD_ERR_ARG, "smd_set_ewald: bad arguments");
    Ctx &c = x->c;
    c.ewald_on = 1;
    c.ew_alpha = alpha;
    c.ew_kcut = kcut;
    c.ew_rc2 = real_cut * real_cut;
    // self and net-charge energies (EwaldForce.cpp:63-79)
    double qsum = 0, q2sum = 0;
    for (int i = 0; i < c.n; i++) {
        qsum += c.h_charge[i];
        q2sum += c.h_charge[i] * c.h_charge[i];
    }
    const double PI = 3.14159265358979323846, SQRT_PI = 1.7724538509055160273;
    c.e_self = -q2sum * alpha / SQRT_PI;
    if (std::fabs(qsum) > 1.0e-5) {
        double vol = c.box.L[0] * c.box.L[1] * c.box.L[2];
        c.e_self += -PI * qsum * qsum / (2.0 * vol * alpha * alpha);
    }
    int r = setup_recip(c);
    if (r) return fail(x, r, "smd_set_ewald: reciprocal set-up failed");
    c.graph_dirty = 1;
    touch(c);
    return SMD_OK;
}

int smd_set_buff(smd_ctx *x, const double *params, double n, double m, double delta, double gamma,
                 double h_factor, int switch_on, double switch_dist, const double *taper_c, double e_lrc,
                 double v_lrc) {
    if (!x || !params || x->c.ntypes == 0 || !(n > m) || !(m > 0))
        return fail(x, SMD_ERR_ARG, "smd_set_buff: bad arguments");
    Ctx &c = x->c;
    const int nt = c.ntypes;
    std::vector<double> p((size_t)nt * nt * 4, 0.0);
    for (int k = 0; k < nt * nt; k++) {
        p[4 * k] = params[2 * k];
        p[4 * k + 1] = params[2 * k + 1];
    }
    CK(cudaMemcpy(c.pair_par, p.data(), p.size() * sizeof(double), cudaMemcpyHostToDevice));
    c.vdw = VDW_BUFF;
    c.buff_on = 1;
    c.buff_n = n; c.buff_m = m; c.buff_delta = delta; c.buff_gamma = gamma; c.buff_h = h_factor;
    c.switch_on = switch_on;
    c.buff_sw = switch_dist;
    for (int q = 0; q < 6; q++) c.buff_c[q] = taper_c ? taper_c[q] : 0.0;
    c.e_lrc = e_lrc;
    c.v_lrc = v_lrc;
    CK(dalloc(&c.vpos4, c.n));
    CK(dalloc(&c.vfixq, c.n));
    CK(dalloc(&c.fv, 3 * (size_t)c.n));
    c.graph_dirty = 1;
    touch(c);
    return SMD_OK;
}

int smd_set_bonded(smd_ctx *x, int nbonds, const int32_t *bonds, int nbond_types, const double *bond_params,
                   int nangles, const int32_t *angles, int nangle_types, const double *angle_params, int form,
                   int ub_on, double k_ub, double l0_ub) {
    if (!x || x->c.n == 0 || nbonds < 0 || nangles < 0 || (nbonds && (!bonds || !bond_params || nbond_types <= 0)) ||
        (nangles && (!angles || !angle_params || nangle_types <= 0)) || (form != 1 && form != 2))
        return fail(x, SMD_ERR_ARG, "smd_set_bonded: bad arguments (form must be 1 harmonic or 2 AMOEBA)");
    Ctx &c = x->c;
    std::vector<int4> b(std::max(nbonds, 1)), g(std::max(nangles, 1));
    for (int k = 0; k < nbonds; k++) {
        const int a1 = bonds[3 * k], a2 = bonds[3 * k + 1], t = bonds[3 * k + 2];
        if (a1 < 0 || a1 >= c.n || a2 < 0 || a2 >= c.n || t < 0 || t >= nbond_types)
            return fail(x, SMD_ERR_ARG, "smd_set_bonded: bond " + std::to_string(k) + " out of range");
        b[k] = make_int4(a1, a2, t, 0);
    }
    for (int k = 0; k < nangles; k++) {
        const int a1 = angles[4 * k], a2 = angles[4 * k + 1], a3 = angles[4 * k + 2], t = angles[4 * k + 3];
        if (a1 < 0 || a1 >= c.n || a2 < 0 || a2 >= c.n || a3 < 0 || a3 >= c.n || t < 0 || t >= nangle_types)
            return fail(x, SMD_ERR_ARG, "smd_set_bonded: angle " + std::to_string(k) + " out of range");
        g[k] = make_int4(a1, a2, a3, t);
    }
    if (ub_on)
        for (int m = 0; m < c.nmol; m++)
            if (c.h_mol_off[m + 1] - c.h_mol_off[m] < 3)
                return fail(x, SMD_ERR_ARG, "smd_set_bonded: the Urey-Bradley term needs molecules of 3 sites");
    std::vector<double2> bp(std::max(nbond_types, 1)), ap(std::max(nangle_types, 1));
    for (int t = 0; t < nbond_types; t++) bp[t] = make_double2(bond_params[2 * t], bond_params[2 * t + 1]);
    for (int t = 0; t < nangle_types; t++) ap[t] = make_double2(angle_params[2 * t], angle_params[2 * t + 1]);
    CK(dalloc(&c.bonds, b.size())); CK(dalloc(&c.angles, g.size()));
    CK(dalloc(&c.bond_par, bp.size())); CK(dalloc(&c.angle_par, ap.size()));
    CK(cudaMemcpy(c.bonds, b.data(), b.size() * sizeof(int4), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.angles, g.data(), g.size() * sizeof(int4), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.bond_par, bp.data(), bp.size() * sizeof(double2), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.angle_par, ap.data(), ap.size() * sizeof(double2), cudaMemcpyHostToDevice));
    c.nbond = nbonds;
    c.nangle = nangles;
    c.bond_form = form;
    c.ub_on = ub_on ? 1 : 0;
    c.ub_k = k_ub;
    c.ub_l0 = l0_ub;
    c.graph_dirty = 1;
    touch(c);
    return SMD_OK;
}

int smd_rdf_setup(smd_ctx *x, int nbins) {
    if (!x || x->c.n == 0 || x->c.box.L[0] <= 0 || nbins <= 0 ||
        (size_t)x->c.ntypes * x->c.ntypes * nbins * sizeof(unsigned int) > 200 * 1024)
        return fail(x, SMD_ERR_ARG, "smd_rdf_setup: nbins must be > 0 with ntypes^2 * nbins * 4 bytes <= 200 KB");
    Ctx &c = x->c;
    CK(cudaSetDevice(c.device));
    const size_t nh = (size_t)c.ntypes * c.ntypes * nbins;
    CK(dalloc(&c.rdf_hist, nh));
    CK(cudaMemsetAsync(c.rdf_hist, 0, nh * sizeof(unsigned long long), c.stream));
    c.rdf_nbins = nbins;
    c.rdf_samples = 0;
    // RDF::init (src/observables/RDF.cpp:47-55): the smallest half box edge
    c.rdf_maxr = std::min(c.box.half[0], std::min(c.box.half[1], c.box.half[2]));
    CK(cudaStreamSynchronize(c.stream));
    return SMD_OK;
}

int smd_rdf_sample(smd_ctx *x) {
    if (!x || !x->c.rdf_hist) return fail(x, SMD_ERR_ARG, "smd_rdf_sample: call smd_rdf_setup first");
    Ctx &c = x->c;
    CK(cudaSetDevice(c.device));
    const int r = rdf_sample(c);
    if (r) return fail(x, r, "smd_rdf_sample: kernel set-up failed");
    return sync_status(x);
}

int smd_rdf_get(smd_ctx *x, uint64_t *hist, double *g, double *r_mid, int64_t *samples) {
    if (!x || !x->c.rdf_hist) return fail(x, SMD_ERR_ARG, "smd_rdf_get: call smd_rdf_setup first");
    Ctx &c = x->c;
    const int nt = c.ntypes, nb = c.rdf_nbins;
    std::vector<unsigned long long> h((size_t)nt * nt * nb);
    CK(cudaMemcpyAsync(h.data(), c.rdf_hist, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       c.stream));
    CK(cudaStreamSynchronize(c.stream));
    if (hist)
        for (size_t k = 0; k < h.size(); k++) hist[k] = h[k];
    if (samples) *samples = c.rdf_samples;
    // RDF::write_result (src/observables/RDF.cpp:146-180)
    const double dr = c.rdf_maxr / nb, vol = c.box.L[0] * c.box.L[1] * c.box.L[2];
    const double pi4dr = 4.0 * 3.14159265358979323846 * dr / vol;
    std::vector<double> per(nt, 0.0);
    for (int i = 0; i < c.n; i++) per[c.h_type[i]] += 1.0;
    int col = 0;
    for (int t1 = 0; t1 < nt; t1++)
        for (int t2 = t1; t2 < nt; t2++, col++)
            for (int k = 0; k < nb; k++) {
                const double r = k * dr + 0.5 * dr;
                if (r_mid && col == 0) r_mid[k] = r;
                if (!g) continue;
                double v = ((double)h[((size_t)t1 * nt + t2) * nb + k] + (double)h[((size_t)t2 * nt + t1) * nb + k]) / pi4dr;
                g[(size_t)col * nb + k] =
                    c.rdf_samples ? 0.5 * v / (r * r * per[t1] * per[t2] * (double)c.rdf_samples) : 0.0;
            }
    return SMD_OK;
}

int smd_averages_reset(smd_ctx *x) {
    if (!x) return SMD_ERR_ARG;
    CK(cudaMemsetAsync(x->c.avg, 0, AVG_COUNT * sizeof(double), x->c.stream));
    CK(cudaStreamSynchronize(x->c.stream));
    return SMD_OK;
}

int smd_get_averages(smd_ctx *x, smd_averages *out) {
    if (!x || !out) return SMD_ERR_ARG;
    double s[AVG_COUNT];
    CK(cudaMemcpyAsync(s, x->c.avg, sizeof(s), cudaMemcpyDeviceToHost, x->c.stream));
    CK(cudaStreamSynchronize(x->c.stream));
    const double n = s[0] > 0 ? s[0] : 1.0;
    out->samples = (int64_t)s[0];
    double *dst[11] = {&out->e_potential, &out->e_potential_sq, &out->e_total, &out->e_total_sq, &out->ke_atom,
                       &out->ke_atom_sq, &out->ke_mol, &out->ke_mol_sq, &out->inv_ke_mol, &out->volume,
                       &out->volume_sq};
    for (int q = 0; q < 11; q++) *dst[q] = s[1 + q] / n;
    for (int q = 0; q < 5; q++) {
        out->atom_stress[q] = s[12 + q] / n;
        out->mol_stress[q] = s[17 + q] / n;
    }
    for (int q = 0; q < 9; q++) {
        out->atom_pressure[q] = s[22 + q] / n;
        out->mol_pressure[q] = s[31 + q] / n;
    }
    return SMD_OK;
}

int smd_set_surface_correct(smd_ctx *x, int on) {
    if (!x || x->c.n == 0 || (on != 0 && on != 1)) return fail(x, SMD_ERR_ARG, "smd_set_surface_correct: bad arguments");
    Ctx &c = x->c;
    if (on && !c.surf_part) {
        CK(dalloc(&c.surf_part, (size_t)SURF_BLOCKS * SURF_SUMS));
        CK(dalloc(&c.surf_tot, SURF_SUMS));
    }
    c.surface_on = on;
    c.graph_dirty = 1;
    touch(c);
    return SMD_OK;
}

int smd_set_multipole(smd_ctx *x, const double *type_mp, const double *polar, double alpha, double kcut,
                      double real_cut, int induction, double ind_cut, double thole_a) {
    if (!x || !type_mp || !polar || !(alpha > 0) || !(kcut > 0) || !(real_cut > 0) || x->c.n == 0)
        return fail(x, SMD_ERR_ARG, "smd_set_multipole: bad arguments");
    Ctx &c = x->c;
    for (int m = 0; m < c.nmol; m++)
        if (c.h_mol_off[m + 1] - c.h_mol_off[m] != 3)
            return fail(x, SMD_ERR_ARG, "smd_set_multipole: molecules must be H O H triples");
    if (real_cut > c.cutoff + 1e-12 || (induction && ind_cut > c.cutoff + 1e-12))
        return fail(x, SMD_ERR_ARG, "smd_set_multipole: real-space and induction cutoffs must not exceed the pair-list cutoff");
    c.mp_on = 1;
    c.ind_on = induction ? 1 : 0;
    c.ew_alpha = alpha;
    c.ew_kcut = kcut;
    c.mp_rc2 = real_cut * real_cut;
    c.ind_cut2 = ind_cut * ind_cut;
    c.thole_a = thole_a;
    c.h_type_polar.assign(polar, polar + c.ntypes);
    CK(dalloc(&c.type_mp, 9 * (size_t)c.ntypes));
    CK(cudaMemcpy(c.type_mp, type_mp, 9 * (size_t)c.ntypes * sizeof(double), cudaMemcpyHostToDevice));
    CK(dalloc(&c.type_polar, c.ntypes));
    CK(cudaMemcpy(c.type_polar, polar, c.ntypes * sizeof(double), cudaMemcpyHostToDevice));
    const size_t n = c.n;
    CK(dalloc(&c.mu, 3 * n)); CK(dalloc(&c.qd, 6 * n)); CK(dalloc(&c.trq, 3 * n));
    CK(dalloc(&c.e0, 3 * n)); CK(dalloc(&c.pind, 3 * n)); CK(dalloc(&c.cgw, 35 * n));
    CK(dalloc(&c.frame, 9 * n));
    CK(dalloc(&c.cg_blk, 81 * (size_t)c.nmol));
    CK(cudaMemset(c.pind, 0, 3 * n * sizeof(double)));
    CK(dalloc(&c.srec, 4 * n));
    CK(cudaMemset(c.srec, 0, 4 * n * sizeof(float4)));
    CK(cudaMemset(c.e0, 0, 3 * n * sizeof(double)));
    int r = setup_cg(c);
    if (r) return fail(x, r, "smd_set_multipole: solver set-up failed");
    const size_t cgb = (size_t)std::max(c.cg_blocks, c.pp_blocks);
    CK(dalloc(&c.cgs, CG_SCAL + CG_TRACE + 16 * cgb));
    CK(cudaMemset(c.cgs, 0, (CG_SCAL + CG_TRACE + 16 * cgb) * sizeof(double)));
    CK(dalloc(&c.cg_bar, 2));
    if (c.ind_on) {
        CK(dalloc(&c.phist, 24 * n));
        CK(cudaMemset(c.flags + 2, 0, 2 * sizeof(int)));
    }
    if (ensure_ind_rows(c)) return fail(x, SMD_ERR_CUDA, "smd_set_multipole: tensor rows: allocation failed");
    r = setup_recip(c);
    if (r) return fail(x, r, "smd_set_multipole: reciprocal set-up failed");
    c.graph_dirty = 1;
    touch(c);
    return SMD_OK;
}

int smd_set_solver(smd_ctx *x, double tol, int max_iter, int guess) {
    if (!x || !(tol > 0) || max_iter <= 0 || guess < 0 || guess > SMD_GUESS_EXTRAP3)
        return fail(x, SMD_ERR_ARG, "smd_set_solver: bad arguments");
    x->c.cg_tol = tol;
    x->c.cg_max_iter = max_iter;
    x->c.cg_guess = guess;
    x->c.graph_dirty = 1;
    touch(x->c);
    return SMD_OK;
}

int smd_set_preconditioner(smd_ctx *x, int kind) {
    if (!x || (kind != SMD_PRECOND_SITE && kind != SMD_PRECOND_MOLECULE))
        return fail(x, SMD_ERR_ARG, "smd_set_preconditioner: kind must be SMD_PRECOND_SITE or SMD_PRECOND_MOLECULE");
    x->c.cg_precond = kind;
    x->c.graph_dirty = 1;
    touch(x->c);
    return SMD_OK;
}

int smd_set_solver_pipelined(smd_ctx *x, int on) {
    if (!x) return fail(x, SMD_ERR_ARG, "smd_set_solver_pipelined: null context");
    if (on < 0 || on > 2) return fail(x, SMD_ERR_ARG, "smd_set_solver_pipelined: mode must be 0, 1 or 2");
    x->c.cg_pipelined = on;
    x->c.graph_dirty = 1;
    touch(x->c);
    return SMD_OK;
}

int smd_set_induction_damping(smd_ctx *x, int form) {
    if (!x) return fail(x, SMD_ERR_ARG, "smd_set_induction_damping: null context");
    if (form < 0 || form > 1) return fail(x, SMD_ERR_ARG, "smd_set_induction_damping: form must be 0 or 1");
    x->c.ind_amoeba = form;
    x->c.graph_dirty = 1;
    touch(x->c);
    return SMD_OK;
}

int smd_mlp_set_tensor_path(smd_ctx *x, int path) {
    if (!x) return fail(x, SMD_ERR_ARG, "smd_mlp_set_tensor_path: null context");
    if (path < 0 || path > 1) return fail(x, SMD_ERR_ARG, "smd_mlp_set_tensor_path: path must be 0 or 1");
    x->c.mlp_tc = path;
    x->c.graph_dirty = 1;
    touch(x->c);
    return SMD_OK;
}

int smd_set_wait_limit(smd_ctx *x, double seconds) {
    if (!x || !(seconds > 0) || seconds > 600)
        return fail(x, SMD_ERR_ARG, "smd_set_wait_limit: the limit must lie in (0, 600] s");
    x->c.wait_ns = (unsigned long long)(seconds * 1e9);
    if (x->c.wait_ns == 0) x->c.wait_ns = 1;
    x->c.graph_dirty = 1;
    return SMD_OK;
}

int smd_test_skip_arrival(smd_ctx *x, int block) {
    if (!x || block < -1 || (block >= 0 && block >= x->c.cg_blocks))
        return fail(x, SMD_ERR_ARG, "smd_test_skip_arrival: block must be -1 or a block of the dipole solve");
    x->c.test_skip_block = block;
    x->c.graph_dirty = 1;
    touch(x->c);
    return SMD_OK;
}

int smd_solver_stats(smd_ctx *x, int *iterations, double *rms_change) {
    if (!x || !x->c.cgs) return fail(x, SMD_ERR_ARG, "smd_solver_stats: no dipole solver");
    double s[2];
    CK(cudaMemcpyAsync(s, x->c.cgs, sizeof(s), cudaMemcpyDeviceToHost, x->c.stream));
    CK(cudaStreamSynchronize(x->c.stream));
    if (iterations) *iterations = (int)s[0];
    if (rms_change) *rms_change = s[1];
    return SMD_OK;
}

int smd_solver_trace(smd_ctx *x, double *rms, int cap, int *count) {
    if (!x || !x->c.cgs || !count || (cap > 0 && !rms)) return fail(x, SMD_ERR_ARG, "smd_solver_trace: bad arguments");
    double s[CG_SCAL + CG_TRACE];
    CK(cudaMemcpyAsync(s, x->c.cgs, sizeof(s), cudaMemcpyDeviceToHost, x->c.stream));
    CK(cudaStreamSynchronize(x->c.stream));
    const int it = std::min((int)s[0], CG_TRACE);
    for (int k = 0; k < std::min(it, cap); k++) rms[k] = s[CG_SCAL + k];
    *count = it;
    return SMD_OK;
}

int smd_get_polarization(smd_ctx *x, double *mu, double *quad, double *e0, double *p) {
    if (!x || !x->c.mp_on) return fail(x, SMD_ERR_ARG, "smd_get_polarization: multipoles not set up");
    Ctx &c = x->c;
    const int n = c.n;
    std::vector<double> h(6 * (size_t)n);
    auto get = [&](const double *src, int comps, double *dst) -> int {
        if (!dst) return SMD_OK;
        CK(cudaMemcpyAsync(h.data(), src, comps * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        CK(cudaStreamSynchronize(c.stream));
        for (int i = 0; i < n; i++)
            for (int d = 0; d < comps; d++) dst[comps * i + d] = h[(size_t)d * n + i];
        return SMD_OK;
    };
    int r;
    if ((r = get(c.mu, 3, mu))) return r;
    if ((r = get(c.qd, 6, quad))) return r;
    if ((r = get(c.e0, 3, e0))) return r;
    if ((r = get(c.pind, 3, p))) return r;
    return SMD_OK;
}

int smd_set_induced(smd_ctx *x, const double *p) {
    if (!x || !p || !x->c.mp_on) return fail(x, SMD_ERR_ARG, "smd_set_induced: multipoles not set up");
    Ctx &c = x->c;
    const int n = c.n;
    std::vector<double> h(3 * (size_t)n);
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) h[(size_t)d * n + i] = p[3 * i + d];
    CK(cudaMemcpy(c.pind, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    touch(c);
    return SMD_OK;
}

// ---- dipole-guess network ------------------------------------------------
int smd_mlp_init(smd_ctx *x, int capacity_frames, unsigned int seed) {
    if (!x || !x->c.ind_on || capacity_frames <= 0)
        return fail(x, SMD_ERR_ARG, "smd_mlp_init: set up the induction model first");
    Ctx &c = x->c;
    int r = mlp_alloc(c, (long long)capacity_frames * c.n, seed);
    if (r) return fail(x, r, "smd_mlp_init: allocation failed");
    c.mlp_ready = 0;
    c.graph_dirty = 1;
    touch(c);
    return SMD_OK;
}

int smd_mlp_dims(int *features, int *params) {
    if (features) *features = mlp_nfeat();
    if (params) *params = mlp_nparam();
    return SMD_OK;
}

int smd_mlp_set_base(smd_ctx *x, int order) {
    if (!x || order < 1 || order > 3) return fail(x, SMD_ERR_ARG, "smd_mlp_set_base: order must be 1, 2 or 3");
    x->c.mlp_base = order;
    x->c.graph_dirty = 1;
    touch(x->c);
    return SMD_OK;
}

int smd_mlp_collect(smd_ctx *x) {
    if (!x || !x->c.mlp_data) return fail(x, SMD_ERR_ARG, "smd_mlp_collect: call smd_mlp_init first");
    Ctx &c = x->c;
    if (c.mlp_rows + c.n > c.mlp_cap) return fail(x, SMD_ERR_ARG, "smd_mlp_collect: training buffer full");
    int cnt = 0;
    CK(cudaMemcpy(&cnt, c.flags + 2, sizeof(int), cudaMemcpyDeviceToHost));
    if (cnt < 2) return fail(x, SMD_ERR_ARG, "smd_mlp_collect: the guess needs 2 stored time steps first");
    launch_mlp_collect(c);
    c.mlp_rows += c.n;
    return sync_status(x);
}

int smd_mlp_train(smd_ctx *x, int epochs, int batch, double lr, unsigned int seed, double *loss) {
    if (!x || !x->c.mlp_data || x->c.mlp_rows == 0 || epochs <= 0 || batch <= 0 || batch > mlp_max_batch())
        return fail(x, SMD_ERR_ARG, "smd_mlp_train: no rows collected or bad batch size");
    Ctx &c = x->c;
    const long long rows = c.mlp_rows;
    if (c.mlp_t == 0) launch_mlp_norm(c);
    std::vector<unsigned int> perm(rows);
    unsigned int *dperm = nullptr;
    CK(cudaMalloc(&dperm, rows * sizeof(unsigned int)));
    unsigned long long s = 0x9E3779B97F4A7C15ull ^ seed;
    for (int ep = 0; ep < epochs; ep++) {
        for (long long k = 0; k < rows; k++) perm[k] = (unsigned int)k;
        for (long long k = rows - 1; k > 0; k--) {  // Fisher-Yates with an xorshift generator
            s ^= s << 13; s ^= s >> 7; s ^= s << 17;
            long long j = (long long)(s % (unsigned long long)(k + 1));
            unsigned int t = perm[k]; perm[k] = perm[j]; perm[j] = t;
        }
        CK(cudaMemcpyAsync(dperm, perm.data(), rows * sizeof(unsigned int), cudaMemcpyHostToDevice, c.stream));
        for (long long r0 = 0; r0 + batch <= rows; r0 += batch) launch_mlp_step(c, dperm, r0, batch, (float)lr, nullptr);
        CK(cudaStreamSynchronize(c.stream));
    }
    if (loss) {  // mean-squared error over (up to) the first max-batch rows of the last order
        const int b = (int)std::min<long long>(rows, mlp_max_batch());
        if (mlp_batch_loss(c, dperm, b, loss)) {
            cudaFree(dperm);
            return fail(x, SMD_ERR_CUDA, "smd_mlp_train: loss evaluation failed");
        }
    }
    cudaFree(dperm);
    c.mlp_ready = 1;
    c.graph_dirty = 1;
    touch(c);
    return sync_status(x);
}

int smd_mlp_params(smd_ctx *x, float *get, const float *set, int *count) {
    if (!x || !x->c.mlp_w) return fail(x, SMD_ERR_ARG, "smd_mlp_params: call smd_mlp_init first");
    Ctx &c = x->c;
    const int np = mlp_nparam(), nf = mlp_nfeat();
    if (count) *count = np + 2 * nf;
    if (get) {
        CK(cudaMemcpy(get, c.mlp_w, np * sizeof(float), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(get + np, c.mlp_norm, 2 * nf * sizeof(float), cudaMemcpyDeviceToHost));
    }
    if (set) {
        CK(cudaMemcpy(c.mlp_w, set, np * sizeof(float), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(c.mlp_norm, set + np, 2 * nf * sizeof(float), cudaMemcpyHostToDevice));
        c.mlp_ready = 1;
        c.mlp_t = std::max(c.mlp_t, 1);
    }
    return SMD_OK;
}

int smd_mlp_eval(smd_ctx *x, const float *feat, int rows, float *out) {
    if (!x || !x->c.mlp_w || !feat || !out || rows <= 0) return fail(x, SMD_ERR_ARG, "smd_mlp_eval: bad arguments");
    Ctx &c = x->c;
    float *dx = nullptr, *dy = nullptr;
    CK(cudaMalloc(&dx, (size_t)rows * mlp_nfeat() * sizeof(float)));
    CK(cudaMalloc(&dy, (size_t)rows * 3 * sizeof(float)));
    CK(cudaMemcpy(dx, feat, (size_t)rows * mlp_nfeat() * sizeof(float), cudaMemcpyHostToDevice));
    launch_mlp_eval(c, rows, dx, dy);
    CK(cudaMemcpyAsync(out, dy, (size_t)rows * 3 * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    int r = sync_status(x);
    cudaFree(dx);
    cudaFree(dy);
    return r;
}

int smd_mlp_gradient(smd_ctx *x, const float *rows_data, int rows, float *grad) {
    if (!x || !x->c.mlp_data || !rows_data || !grad || rows <= 0 || rows > mlp_max_batch() ||
        rows > x->c.mlp_cap)
        return fail(x, SMD_ERR_ARG, "smd_mlp_gradient: bad arguments");
    Ctx &c = x->c;
    const int w = mlp_nfeat() + 3;
    CK(cudaMemcpy(c.mlp_data, rows_data, (size_t)rows * w * sizeof(float), cudaMemcpyHostToDevice));
    c.mlp_rows = rows;
    std::vector<unsigned int> perm(rows);
    for (int k = 0; k < rows; k++) perm[k] = k;
    unsigned int *dperm = nullptr;
    float *dg = nullptr;
    CK(cudaMalloc(&dperm, rows * sizeof(unsigned int)));
    CK(cudaMalloc(&dg, mlp_nparam() * sizeof(float)));
    CK(cudaMemcpy(dperm, perm.data(), rows * sizeof(unsigned int), cudaMemcpyHostToDevice));
    launch_mlp_step(c, dperm, 0, rows, 0.f, dg);
    CK(cudaMemcpyAsync(grad, dg, mlp_nparam() * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    int r = sync_status(x);
    cudaFree(dperm);
    cudaFree(dg);
    c.mlp_rows = 0;
    return r;
}

int smd_mlp_features(smd_ctx *x, float *feat) {
    if (!x || !x->c.mlp_x || !feat) return fail(x, SMD_ERR_ARG, "smd_mlp_features: call smd_mlp_init first");
    Ctx &c = x->c;
    launch_mlp_features(c);
    CK(cudaMemcpyAsync(feat, c.mlp_x, (size_t)c.n * mlp_nfeat() * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
    return sync_status(x);
}

int smd_set_precision(smd_ctx *x, int mode) {
    if (!x || (mode != SMD_PREC_FP64 && mode != SMD_PREC_MIXED))
        return fail(x, SMD_ERR_ARG, "smd_set_precision: unknown mode");
    x->c.precision = mode;
    if (x->c.n > 0 && x->c.pos4) launch_fixq(x->c);
    x->c.graph_dirty = 1;
    touch(x->c);
    return SMD_OK;
}

int smd_set_reference_forms(smd_ctx *x, int on) {
    if (!x || (on != 0 && on != 1)) return fail(x, SMD_ERR_ARG, "smd_set_reference_forms: on must be 0 or 1");
    x->c.reference_forms = on;
    x->c.graph_dirty = 1;
    touch(x->c);
    return SMD_OK;
}

int smd_set_tuning(smd_ctx *x, int tpp) {
    if (!x) return SMD_ERR_ARG;
    if (tpp == 0) tpp = 8;
    if (tpp < 1 || tpp > 32 || (tpp & (tpp - 1)))
        return fail(x, SMD_ERR_ARG, "smd_set_tuning: threads per site must be a power of two <= 32");
    x->c.tpp = tpp;
    x->c.graph_dirty = 1;
    touch(x->c);
    return SMD_OK;
}

int smd_upload_positions(smd_ctx *x, const double *pos) {
    if (!x || !pos || x->c.n == 0) return fail(x, SMD_ERR_ARG, "smd_upload_positions: bad arguments");
    Ctx &c = x->c;
    for (int i = 0; i < 3 * c.n; i++)
        if (!std::isfinite(pos[i]))
            return fail(x, SMD_ERR_NAN, "smd_upload_positions: non-finite coordinate of site " + std::to_string(i / 3));
    std::vector<double4> p(c.n);
    for (int i = 0; i < c.n; i++)
        p[i] = make_double4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], (double)c.h_type[i]);
    if (c.list_built && c.ip.strain_rate == 0.0) {
        // the list stays valid while every site has moved less than half the
        // skin since the last rebuild: the upload adds each site's minimum-image
        // displacement and raises the rebuild flag past that, as a step does
        if (!c.upload4) CK(dalloc(&c.upload4, c.n));
        CK(cudaMemcpyAsync(c.upload4, p.data(), c.n * sizeof(double4), cudaMemcpyHostToDevice, c.stream));
        launch_upload_positions(c);
    } else {
        CK(cudaMemcpyAsync(c.pos4, p.data(), c.n * sizeof(double4), cudaMemcpyHostToDevice, c.stream));
        CK(cudaMemsetAsync(c.disp4, 0, c.n * sizeof(double4), c.stream));
        int one = 1;  // the next step rebuilds the pair list from these positions
        CK(cudaMemcpyAsync(c.flags, &one, sizeof(int), cudaMemcpyHostToDevice, c.stream));
    }
    launch_fixq(c);
    // realPos starts as these positions (smd_upload_real_positions may set it)
    CK(cudaMemsetAsync(c.wrap, 0, 3 * (size_t)c.nmol * sizeof(double), c.stream));
    c.h_real_off.clear();
    CK(cudaStreamSynchronize(c.stream));
    c.list_valid = 0;   // smd_get_pairs builds a fresh list from these positions
    touch(c);
    return SMD_OK;
}

int smd_upload_real_positions(smd_ctx *x, const double *real) {
    if (!x || !real || x->c.n == 0 || !x->c.pos4) return fail(x, SMD_ERR_ARG, "smd_upload_real_positions: bad arguments");
    Ctx &c = x->c;
    std::vector<double> p(3 * (size_t)c.n);
    int r = smd_download_state(x, p.data(), nullptr, nullptr);
    if (r) return r;
    std::vector<double> w(3 * (size_t)c.nmol);
    CK(cudaMemcpy(w.data(), c.wrap, w.size() * sizeof(double), cudaMemcpyDeviceToHost));
    c.h_real_off.assign(3 * (size_t)c.n, 0.0);
    for (int i = 0; i < c.n; i++)
        for (int d = 0; d < 3; d++) {
            if (!std::isfinite(real[3 * i + d]))
                return fail(x, SMD_ERR_NAN, "smd_upload_real_positions: non-finite coordinate");
            c.h_real_off[3 * i + d] = real[3 * i + d] - (p[3 * i + d] - w[(size_t)d * c.nmol + c.h_mol[i]]);
        }
    return SMD_OK;
}

int smd_download_real_positions(smd_ctx *x, double *real) {
    if (!x || !real || x->c.n == 0) return fail(x, SMD_ERR_ARG, "smd_download_real_positions: bad arguments");
    Ctx &c = x->c;
    int r = smd_download_state(x, real, nullptr, nullptr);
    if (r) return r;
    std::vector<double> w(3 * (size_t)c.nmol);
    CK(cudaMemcpy(w.data(), c.wrap, w.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int i = 0; i < c.n; i++)
        for (int d = 0; d < 3; d++) {
            real[3 * i + d] -= w[(size_t)d * c.nmol + c.h_mol[i]];
            if (!c.h_real_off.empty()) real[3 * i + d] += c.h_real_off[3 * i + d];
        }
    return SMD_OK;
}

int smd_get_integrator_state(smd_ctx *x, double *state) {
    if (!x || !state || !x->c.scal) return SMD_ERR_ARG;
    CK(cudaMemcpyAsync(state, x->c.scal, SC_NSCAL * sizeof(double), cudaMemcpyDeviceToHost, x->c.stream));
    CK(cudaStreamSynchronize(x->c.stream));
    return SMD_OK;
}

int smd_set_integrator_state(smd_ctx *x, const double *state) {
    if (!x || !state || !x->c.scal) return SMD_ERR_ARG;
    for (int q = 0; q < SC_NSCAL; q++)
        if (!std::isfinite(state[q])) return fail(x, SMD_ERR_NAN, "smd_set_integrator_state: non-finite value");
    CK(cudaMemcpyAsync(x->c.scal, state, SC_NSCAL * sizeof(double), cudaMemcpyHostToDevice, x->c.stream));
    CK(cudaStreamSynchronize(x->c.stream));
    touch(x->c);
    return SMD_OK;
}

int smd_upload_velocities(smd_ctx *x, const double *vel, const double *vtminus) {
    if (!x || !vel || x->c.n == 0) return fail(x, SMD_ERR_ARG, "smd_upload_velocities: bad arguments");
    Ctx &c = x->c;
    for (int i = 0; i < 3 * c.n; i++)
        if (!std::isfinite(vel[i]) || (vtminus && !std::isfinite(vtminus[i])))
            return fail(x, SMD_ERR_NAN, "smd_upload_velocities: non-finite velocity of site " + std::to_string(i / 3));
    std::vector<double4> v(c.n), vm(c.n);
    for (int i = 0; i < c.n; i++) {
        v[i] = make_double4(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2], 1.0 / c.h_mass[i]);
        const double *s = vtminus ? vtminus : vel;
        vm[i] = make_double4(s[3 * i], s[3 * i + 1], s[3 * i + 2], c.h_mass[i]);
    }
    CK(cudaMemcpyAsync(c.vel4, v.data(), c.n * sizeof(double4), cudaMemcpyHostToDevice, c.stream));
    CK(cudaMemcpyAsync(c.vtm4, vm.data(), c.n * sizeof(double4), cudaMemcpyHostToDevice, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return SMD_OK;
}

int smd_download_state(smd_ctx *x, double *pos, double *vel, double *vtminus) {
    if (!x || x->c.n == 0) return fail(x, SMD_ERR_ARG, "smd_download_state: bad arguments");
    Ctx &c = x->c;
    std::vector<double4> h(c.n);
    double *outs[3] = {pos, vel, vtminus};
    double4 *srcs[3] = {c.pos4, c.vel4, c.vtm4};
    for (int q = 0; q < 3; q++) {
        if (!outs[q]) continue;
        CK(cudaMemcpyAsync(h.data(), srcs[q], c.n * sizeof(double4), cudaMemcpyDeviceToHost, c.stream));
        CK(cudaStreamSynchronize(c.stream));
        for (int i = 0; i < c.n; i++) {
            outs[q][3 * i] = h[i].x;
            outs[q][3 * i + 1] = h[i].y;
            outs[q][3 * i + 2] = h[i].z;
        }
    }
    return SMD_OK;
}

int smd_compute_forces(smd_ctx *x, uint32_t terms, double *force, double *energy, double *virial) {
    if (!x || x->c.n == 0 || x->c.box.L[0] <= 0) return fail(x, SMD_ERR_ARG, "smd_compute_forces: system not set up");
    Ctx &c = x->c;
    CK(cudaSetDevice(c.device));
    if (force && !c.fout) CK(dalloc(&c.fout, 3 * (size_t)c.n));   // once per context
    return compute_forces_into(x, terms, c.fout, force, energy, virial);
}

}  // extern "C"

extern "C" {

int smd_compute_forces_noalloc(smd_ctx *x, uint32_t terms, double *force, double *energy, double *virial) {
    if (!x || x->c.n == 0 || x->c.box.L[0] <= 0)
        return fail(x, SMD_ERR_ARG, "smd_compute_forces_noalloc: system not set up");
    Ctx &c = x->c;
    if (c.n > NOALLOC_MAX_SITES)
        return fail(x, SMD_ERR_ARG, "smd_compute_forces_noalloc: " + std::to_string(c.n) +
                                        " sites exceed the static scratch of " +
                                        std::to_string(NOALLOC_MAX_SITES) + " sites");
    if (c.device < 0 || c.device >= NOALLOC_MAX_DEVICES)
        return fail(x, SMD_ERR_ARG, "smd_compute_forces_noalloc: device index out of range");
    CK(cudaSetDevice(c.device));
    double *dforce = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[c.device]) {
            // once per device, with that device current
            void *a = nullptr;
            CK(cudaGetSymbolAddress(&a, g_noalloc_force));
            g_noalloc_addr[c.device] = (double *)a;
        }
        dforce = g_noalloc_addr[c.device];
    }
    return compute_forces_into(x, terms, dforce, force, energy, virial);
}

int smd_get_pairs(smd_ctx *x, int32_t *pairs, int64_t cap, int64_t *count) {
    if (!x || !count || x->c.n == 0) return fail(x, SMD_ERR_ARG, "smd_get_pairs: bad arguments");
    Ctx &c = x->c;
    if (!c.list_valid) {
        CK(cudaMemsetAsync(c.status, 0, sizeof(unsigned), c.stream));
        launch_nlist(c, true);
        c.list_valid = 1;
        int rs = sync_status(x);
        if (rs) return rs;
    }
    std::vector<int> nn(c.n);
    std::vector<int> nb((size_t)c.pl.max_nbr * c.n);
    CK(cudaMemcpy(nn.data(), c.pl.nnbr, c.n * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(nb.data(), c.pl.nbr, nb.size() * sizeof(int), cudaMemcpyDeviceToHost));
    int64_t k = 0;
    for (int i = 0; i < c.n; i++)
        for (int q = 0; q < nn[i]; q++) {
            int j = nb[(size_t)q * c.n + i] & 0x7fffffff;
            if (i < j) {
                if (pairs && k < cap) { pairs[2 * k] = i; pairs[2 * k + 1] = j; }
                k++;
            }
        }
    *count = k;
    return SMD_OK;
}

int smd_ewald_nk(smd_ctx *x, int *nk) {
    if (!x || !nk) return SMD_ERR_ARG;
    const int r = recip_nk(x->c, nk);
    return r ? fail(x, r, "smd_ewald_nk: reading the k count failed") : SMD_OK;
}

int smd_set_integrator(smd_ctx *x, const smd_integrator_params *p) {
    if (!x || !p || !(p->timestep > 0) || x->c.n == 0)
        return fail(x, SMD_ERR_ARG, "smd_set_integrator: bad arguments");
    if (p->constraint != 0 && p->constraint != 2)
        return fail(x, SMD_ERR_ARG, "smd_set_integrator: constraint must be 0 (none) or 2 (SHAKE)");
    if (p->constraint == 2 && !x->c.clen2)
        return fail(x, SMD_ERR_ARG, "smd_set_integrator: SHAKE needs smd_set_constraints first");
    if (p->constraint == 2 && (p->shake_max_iter <= 0 || !(p->shake_tol > 0)))
        return fail(x, SMD_ERR_ARG, "smd_set_integrator: SHAKE tolerance and maxCount must be > 0");
    if (p->long_steps > 1)
        return fail(x, SMD_ERR_ARG, "smd_set_integrator: long_steps > 1 not supported");
    if (p->thermostat < SMD_THERMO_NONE || p->thermostat > SMD_THERMO_NH_CHAIN)
        return fail(x, SMD_ERR_ARG, "smd_set_integrator: unknown thermostat");
    if (p->thermostat == SMD_THERMO_NH_CHAIN && (p->constraint != 0 || !(p->coupl_const > 0)))
        return fail(x, SMD_ERR_ARG, "smd_set_integrator: the chain integrator needs tau > 0 and no constraints");
    if (p->strain_rate != 0.0) {
        if (p->thermostat != SMD_THERMO_NH_CHAIN)
            return fail(x, SMD_ERR_ARG, "smd_set_integrator: SLLOD shear runs with the chain integrator");
        if (x->c.mp_on || x->c.vdw == VDW_BUFF || x->c.surface_on)
            return fail(x, SMD_ERR_ARG,
                        "smd_set_integrator: SLLOD shear supports the LJ / Mie / BMH pair terms, point-charge "
                        "Ewald and bonded terms (no multipoles, buffered 14-7 or surface correction)");
    }
    Ctx &c = x->c;
    const bool was_sheared = c.integrator_ready && c.ip.strain_rate != 0.0;
    c.ip = *p;
    // the sheared cell search moves a 4-cell x window across the y boundary
    if (p->strain_rate != 0.0 && c.grid.use_cells && c.grid.n[0] < 4) c.grid.use_cells = 0;
    if (c.ip.atom_ndf <= 0) c.ip.atom_ndf = 3 * c.n - 3;
    if (c.ip.mol_ndf <= 0) c.ip.mol_ndf = 3 * c.nmol - 3;
    c.integrator_ready = 1;
    // the point-charge reciprocal sum under shear takes its k list from the
    // offset (and back to the fixed list without shear)
    if (c.ewald_on && (was_sheared || p->strain_rate != 0.0)) {
        const int r = setup_recip(c);
        if (r) return fail(x, r, "smd_set_integrator: reciprocal set-up failed");
    }
    c.graph_dirty = 1;
    touch(c);
    return SMD_OK;
}

int smd_set_constraints(smd_ctx *x, const double *len2) {
    if (!x || !len2 || x->c.nmol == 0) return fail(x, SMD_ERR_ARG, "smd_set_constraints: bad arguments");
    Ctx &c = x->c;
    for (int m = 0; m < c.nmol; m++) {
        int ns = c.h_mol_off[m + 1] - c.h_mol_off[m];
        if (ns > 8) return fail(x, SMD_ERR_ARG, "smd_set_constraints: molecules of more than 8 sites");
        for (int q = 0; q < 3; q++)
            if (ns > 1 && !(len2[3 * m + q] > 0))
                return fail(x, SMD_ERR_ARG, "smd_set_constraints: squared lengths must be > 0");
    }
    CK(dalloc(&c.clen2, 3 * (size_t)c.nmol));
    CK(cudaMemcpy(c.clen2, len2, 3 * (size_t)c.nmol * sizeof(double), cudaMemcpyHostToDevice));
    c.graph_dirty = 1;
    touch(c);
    return SMD_OK;
}

// new_start: LFIntegrator::start's half-step velocities from the forces;
// otherwise the uploaded ones are kept (the run that continues from
// state.in and vtMinus.in, LFIntegrator.cpp:187-192)
static int integrator_begin(smd_ctx *x, bool new_start) {
    if (!x || !x->c.integrator_ready) return fail(x, SMD_ERR_ARG, "smd_integrator_start: call smd_set_integrator first");
    Ctx &c = x->c;
    CK(cudaSetDevice(c.device));
    CK(cudaMemsetAsync(c.status, 0, sizeof(unsigned), c.stream));
    CK(cudaMemsetAsync(c.obs, 0, sizeof(smd_observables), c.stream));
    CK(cudaMemsetAsync(c.avg, 0, AVG_COUNT * sizeof(double), c.stream));   // averages of this run
    CK(cudaMemsetAsync(c.ticket, 0, sizeof(unsigned), c.stream));
    // the dipole history of the guess starts afresh (uploads keep it: the
    // solve converges to its tolerance from any start)
    CK(cudaMemsetAsync(c.flags + 2, 0, 2 * sizeof(int), c.stream));   // step count and the push's ticket
    if (c.npt) {
        // NHIntegrator's NpT run: pair terms only (the reciprocal sums keep
        // their k-vectors of one box), no constraints (the reference stops
        // there too, NHIntegrator.cpp:604-607), FP64
        if (c.ip.thermostat != SMD_THERMO_NH_CHAIN || c.ip.strain_rate != 0.0 || c.ewald_on || c.mp_on ||
            has_bonded(c) || c.precision != SMD_PREC_FP64 || c.vdw == VDW_BUFF || c.vdw == VDW_SAAP ||
            c.wolf_on)
            return fail(x, SMD_ERR_ARG,
                        "smd_integrator_start: the barostat runs with the chain integrator on pair terms in FP64");
        CK(cudaMemcpy(c.dbox, &c.box, sizeof(Box), cudaMemcpyHostToDevice));
        setup_grid(c, c.want_cells);
        int r = alloc_list(x);
        if (r) return r;
        const double vol = c.box.L[0] * c.box.L[1] * c.box.L[2];
        c.npt_lrc_k = c.e_lrc * vol;
        c.npt_smin = 0.0;
        if (c.grid.use_cells)
            for (int d = 0; d < 3; d++)
                c.npt_smin = std::max(c.npt_smin, c.grid.n[d] * (c.cutoff + c.cut_buffer) / c.box.L[d]);
    }
    if (c.ip.strain_rate != 0.0 && (c.mp_on || c.vdw == VDW_BUFF || c.surface_on))
        return fail(x, SMD_ERR_ARG,
                    "smd_integrator_start: SLLOD shear takes no multipoles, buffered 14-7 or surface correction");
    launch_nlist(c, true);
    c.list_valid = 1;
    CK(cudaMemsetAsync(c.acc, 0, ACC_COUNT * sizeof(long long), c.stream));
    if (c.ip.thermostat == SMD_THERMO_NH_CHAIN) {
        launch_nhc_start(c);   // delta = 0 before the first list and forces
        // the barostat at rest; molVirt = -P until the first forces
        // (Integrator.cpp:44-46), vlog = 0 (NHIntegrator.cpp:120)
        const double bs[5] = {0.0, c.npt ? -c.npt_press : 0.0, 1.0, c.ip.timestep,
                              c.box.L[0] * c.box.L[1] * c.box.L[2]};
        CK(cudaMemcpyAsync(c.scal + SC_VLOG, bs, sizeof(bs), cudaMemcpyHostToDevice, c.stream));
        launch_nlist(c, true);
        CK(cudaMemsetAsync(c.acc, 0, ACC_COUNT * sizeof(long long), c.stream));
        enqueue_forces(c);
        CK(cudaMemsetAsync(c.acc, 0, ACC_COUNT * sizeof(long long), c.stream));
    } else {
        enqueue_forces(c);
        if (new_start) launch_start_velocities(c);
    }
    // numUpdates counts the rebuilds of the run, not the start's
    // (LFIntegrator.cpp:307-341): the build count restarts here
    CK(cudaMemsetAsync(c.flags + 1, 0, sizeof(int), c.stream));
    c.steps_done = 0;
    touch(c);
    return sync_status(x);
}

int smd_integrator_start(smd_ctx *x) { return integrator_begin(x, true); }

int smd_integrator_resume(smd_ctx *x) { return integrator_begin(x, false); }

// after barostat steps: the host copy of the box and the tail correction
// follow the device's (the cell grid stays laid out for the box it was
// built for; the kernels scale it)
static void sync_npt_box(Ctx &c) {
    Box b;
    if (cudaMemcpy(&b, c.dbox, sizeof(Box), cudaMemcpyDeviceToHost) != cudaSuccess) return;
    c.box = b;
    const double vol = b.L[0] * b.L[1] * b.L[2];
    c.e_lrc = c.npt_lrc_k / vol;
    c.v_lrc = -2.0 * c.e_lrc;
}

int smd_run(smd_ctx *x, int nsteps) {
    if (!x || !x->c.integrator_ready || nsteps < 0) return fail(x, SMD_ERR_ARG, "smd_run: integrator not set");
    Ctx &c = x->c;
    CK(cudaSetDevice(c.device));
    if (c.graph_dirty || !c.step_graph) {
        if (c.step_graph) { cudaGraphExecDestroy(c.step_graph); c.step_graph = nullptr; }
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
        enqueue_step(c);
        CK(cudaStreamEndCapture(c.stream, &g));
        cudaError_t e = cudaGraphInstantiate(&c.step_graph, g, 0);
        cudaGraphDestroy(g);
        CK(e);
        c.graph_dirty = 0;
    }
    for (int s = 0; s < nsteps; s++) CK(cudaGraphLaunch(c.step_graph, c.stream));
    c.steps_done += nsteps;
    if (nsteps > 0) touch(c);
    int r = sync_status(x);
    if (c.npt) sync_npt_box(c);
    return r;
}

int smd_profile_stages(smd_ctx *x, int reps, double *out) {
    if (!x || !out || reps <= 0 || !x->c.integrator_ready)
        return fail(x, SMD_ERR_ARG, "smd_profile_stages: set up the integrator first");
    Ctx &c = x->c;
    CK(cudaSetDevice(c.device));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    // keep the state: the integrate stage runs on a copy of the step inputs
    std::vector<long long> save_acc(ACC_COUNT);
    float ms = 0;
    auto timed = [&](auto &&fn) -> double {
        fn();  // warm
        cudaEventRecord(e0, c.stream);
        for (int r = 0; r < reps; r++) fn();
        cudaEventRecord(e1, c.stream);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        return (double)ms / reps;
    };
    out[0] = timed([&] { launch_pair(c); });
    out[1] = c.ewald_on ? timed([&] { launch_recip(c); }) : 0.0;
    // integrate on scratch copies of the moving state
    size_t nb = (size_t)c.n * sizeof(double4);
    double4 *b_pos, *b_vel, *b_vtm, *b_disp;
    CK(cudaMalloc(&b_pos, nb)); CK(cudaMalloc(&b_vel, nb));
    CK(cudaMalloc(&b_vtm, nb)); CK(cudaMalloc(&b_disp, nb));
    CK(cudaMemcpyAsync(b_pos, c.pos4, nb, cudaMemcpyDeviceToDevice, c.stream));
    CK(cudaMemcpyAsync(b_vel, c.vel4, nb, cudaMemcpyDeviceToDevice, c.stream));
    CK(cudaMemcpyAsync(b_vtm, c.vtm4, nb, cudaMemcpyDeviceToDevice, c.stream));
    CK(cudaMemcpyAsync(b_disp, c.disp4, nb, cudaMemcpyDeviceToDevice, c.stream));
    smd_observables o_save;
    CK(cudaMemcpyAsync(&o_save, c.obs, sizeof(o_save), cudaMemcpyDeviceToHost, c.stream));
    double sc_save[8];
    CK(cudaMemcpyAsync(sc_save, c.scal, sizeof(sc_save), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    std::swap(c.pos4, b_pos); std::swap(c.vel4, b_vel); std::swap(c.vtm4, b_vtm); std::swap(c.disp4, b_disp);
    out[2] = timed([&] { launch_integrate(c); });
    std::swap(c.pos4, b_pos); std::swap(c.vel4, b_vel); std::swap(c.vtm4, b_vtm); std::swap(c.disp4, b_disp);
    CK(cudaMemcpyAsync(c.obs, &o_save, sizeof(o_save), cudaMemcpyHostToDevice, c.stream));
    CK(cudaMemcpyAsync(c.scal, sc_save, sizeof(sc_save), cudaMemcpyHostToDevice, c.stream));
    out[3] = timed([&] { launch_nlist(c, true); });
    for (int q = 4; q < 12; q++) out[q] = 0.0;
    if (c.mp_on) {
        out[4] = timed([&] { launch_frames(c); });
        const bool fused = polar_short_fused(c);
        if (!fused) out[5] = timed([&] { launch_mp_short(c); });
        if (!c.ind_on) out[6] = timed([&] { launch_mp_long(c); });
        if (c.ind_on) {
            const int guess = c.cg_guess;
            if (guess == 0) {
                out[7] = timed([&] { launch_ind_solve(c); });
            } else {
                // a warm start must start from the same dipoles every time
                // (a device copy: its time is a few microseconds of the stage)
                const size_t pb = 3 * (size_t)c.n * sizeof(double);
                double *p0 = nullptr;
                CK(cudaMalloc(&p0, pb));
                CK(cudaMemcpyAsync(p0, c.pind, pb, cudaMemcpyDeviceToDevice, c.stream));
                out[7] = timed([&] {
                    cudaMemcpyAsync(c.pind, p0, pb, cudaMemcpyDeviceToDevice, c.stream);
                    launch_ind_solve(c);
                });
                CK(cudaStreamSynchronize(c.stream));
                cudaFree(p0);
            }
            // with the fused pass the multipole real space is part of this stage
            out[8] = timed([&] { if (fused) launch_polar_short(c); else launch_ind_short(c); });
            out[9] = timed([&] { launch_polar_long(c); });
            // the solve's two parts: the permanent field with the tensor rows,
            // the preconditioner blocks and the start dipoles; then the PCG
            // kernel alone, each time from the same start dipoles (a device
            // copy of 3N doubles, about a microsecond, inside its time)
            out[10] = timed([&] { launch_ind_field(c); });
            {
                const size_t pb = 3 * (size_t)c.n * sizeof(double);
                double *p0 = nullptr;
                CK(cudaMalloc(&p0, pb));
                CK(cudaMemcpyAsync(p0, c.pind, pb, cudaMemcpyDeviceToDevice, c.stream));
                out[11] = timed([&] {
                    cudaMemcpyAsync(c.pind, p0, pb, cudaMemcpyDeviceToDevice, c.stream);
                    launch_ind_cg(c);
                });
                CK(cudaStreamSynchronize(c.stream));
                cudaFree(p0);
            }
        }
    }
    // forces for the current positions again, accumulators clear
    CK(cudaMemsetAsync(c.acc, 0, ACC_COUNT * sizeof(long long), c.stream));
    enqueue_forces(c);
    CK(cudaMemsetAsync(c.acc, 0, ACC_COUNT * sizeof(long long), c.stream));
    CK(cudaStreamSynchronize(c.stream));
    cudaFree(b_pos); cudaFree(b_vel); cudaFree(b_vtm); cudaFree(b_disp);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    touch(c);
    return sync_status(x);
}

int smd_step_kernel_count(smd_ctx *x, int *count) {
    if (!x || !count) return SMD_ERR_ARG;
    Ctx &c = x->c;
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
    enqueue_step(c);
    CK(cudaStreamEndCapture(c.stream, &g));
    size_t nn = 0;
    CK(cudaGraphGetNodes(g, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    CK(cudaGraphGetNodes(g, nodes.data(), &nn));
    int k = 0;
    for (auto nd : nodes) {
        cudaGraphNodeType t;
        cudaGraphNodeGetType(nd, &t);
        if (t == cudaGraphNodeTypeKernel) k++;
    }
    cudaGraphDestroy(g);
    *count = k;
    return SMD_OK;
}

int smd_run_timed(smd_ctx *x, int nsteps, double *device_ms) {
    if (!x || !device_ms || !x->c.integrator_ready || nsteps < 0)
        return fail(x, SMD_ERR_ARG, "smd_run_timed: integrator not set");
    Ctx &c = x->c;
    CK(cudaSetDevice(c.device));
    if (c.graph_dirty || !c.step_graph) {
        int r = smd_run(x, 0);
        if (r) return r;
    }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaStreamSynchronize(c.stream));
    CK(cudaEventRecord(e0, c.stream));
    for (int s = 0; s < nsteps; s++) CK(cudaGraphLaunch(c.step_graph, c.stream));
    CK(cudaEventRecord(e1, c.stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    *device_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c.steps_done += nsteps;
    if (nsteps > 0) touch(c);
    int r = sync_status(x);
    if (c.npt) sync_npt_box(c);
    return r;
}

int smd_get_observables(smd_ctx *x, smd_observables *out) {
    if (!x || !out) return SMD_ERR_ARG;
    Ctx &c = x->c;
    CK(cudaMemcpyAsync(out, c.obs, sizeof(smd_observables), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return SMD_OK;
}

int smd_set_series_capacity(smd_ctx *x, int cap) {
    if (!x || cap < 0) return SMD_ERR_ARG;
    Ctx &c = x->c;
    if (c.series) { cudaFree(c.series); c.series = nullptr; }
    c.series_cap = cap;
    if (cap > 0) {
        CK(cudaMalloc(&c.series, (size_t)cap * 5 * sizeof(double)));
        CK(cudaMemset(c.series, 0, (size_t)cap * 5 * sizeof(double)));
    }
    c.graph_dirty = 1;
    touch(c);
    return SMD_OK;
}

int smd_get_series(smd_ctx *x, double *out, int cap, int *count) {
    if (!x || !out || !count) return SMD_ERR_ARG;
    Ctx &c = x->c;
    smd_observables o;
    int r = smd_get_observables(x, &o);
    if (r) return r;
    long long steps = o.step;
    int have = (int)std::min<long long>(steps, c.series_cap);
    have = std::min(have, cap);
    std::vector<double> all((size_t)c.series_cap * 5);
    if (c.series_cap) CK(cudaMemcpy(all.data(), c.series, all.size() * sizeof(double), cudaMemcpyDeviceToHost));
    // oldest first
    for (int k = 0; k < have; k++) {
        long long stepno = steps - have + k;  // 0-based step index
        long long slot = stepno % c.series_cap;
        for (int q = 0; q < 5; q++) out[5 * k + q] = all[slot * 5 + q];
    }
    *count = have;
    return SMD_OK;
}


/* ---- batched replicas --------------------------------------------------- */
}  // extern "C"

struct smd_batch {
    int device = 0;
    std::vector<smd_ctx *> reps;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    int dirty = 1;
    std::string err;
};

namespace {
int bfail(smd_batch *b, int code, const std::string &msg) {
    if (b) b->err = msg;
    return code;
}
#define BCK(call)                                                                              \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return bfail(b, SMD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// every replica's step as one branch of one graph: fork from the batch
// stream, each replica's kernels on its own stream, join back
int batch_build(smd_batch *b) {
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    cudaGraph_t g;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaEventRecord(b->fork, b->stream);
    for (size_t r = 0; r < b->reps.size(); r++) {
        Ctx &c = b->reps[r]->c;
        cudaStreamWaitEvent(c.stream, b->fork, 0);
        enqueue_step(c);
        cudaEventRecord(b->join[r], c.stream);
        cudaStreamWaitEvent(b->stream, b->join[r], 0);
    }
    BCK(cudaStreamEndCapture(b->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    BCK(e);
    b->dirty = 0;
    return SMD_OK;
}

int batch_status(smd_batch *b) {
    BCK(cudaStreamSynchronize(b->stream));
    for (size_t r = 0; r < b->reps.size(); r++) {
        const int rc = sync_status(b->reps[r]);
        if (rc) return bfail(b, rc, "replica " + std::to_string(r) + ": " + b->reps[r]->c.err);
    }
    return SMD_OK;
}
}  // namespace

extern "C" {

int smd_batch_create(smd_ctx *const *ctxs, int count, smd_batch **out) {
    if (!out || !ctxs || count <= 0) return SMD_ERR_ARG;
    *out = nullptr;
    smd_batch *b = new (std::nothrow) smd_batch();
    if (!b) return SMD_ERR_ARG;
    b->device = ctxs[0] ? ctxs[0]->c.device : 0;
    for (int r = 0; r < count; r++) {
        if (!ctxs[r] || !ctxs[r]->c.integrator_ready || ctxs[r]->c.device != b->device) {
            delete b;
            return SMD_ERR_ARG;
        }
        b->reps.push_back(ctxs[r]);
    }
    if (cudaSetDevice(b->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) {
        delete b;
        return SMD_ERR_CUDA;
    }
    b->join.assign(count, nullptr);
    for (int r = 0; r < count; r++)
        if (cudaEventCreateWithFlags(&b->join[r], cudaEventDisableTiming) != cudaSuccess) {
            smd_batch_destroy(b);
            return SMD_ERR_CUDA;
        }
    *out = b;
    return SMD_OK;
}

void smd_batch_destroy(smd_batch *b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (cudaEvent_t e : b->join)
        if (e) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

const char *smd_batch_last_error(const smd_batch *b) { return b ? b->err.c_str() : "null batch"; }

int smd_batch_autotune(smd_batch *b, int reps, int32_t *tpp_out) {
    if (!b || reps <= 0) return SMD_ERR_ARG;
    BCK(cudaSetDevice(b->device));
    cudaEvent_t e0, e1;
    BCK(cudaEventCreate(&e0));
    BCK(cudaEventCreate(&e1));
    const int cand[6] = {1, 2, 4, 8, 16, 32};
    for (size_t r = 0; r < b->reps.size(); r++) {
        Ctx &c = b->reps[r]->c;
        float best = 1e30f;
        int best_t = c.tpp;
        for (int q = 0; q < 6; q++) {
            c.tpp = cand[q];
            launch_pair(c);   // warm
            cudaEventRecord(e0, c.stream);
            for (int k = 0; k < reps; k++) launch_pair(c);
            cudaEventRecord(e1, c.stream);
            BCK(cudaEventSynchronize(e1));
            float ms = 0;
            BCK(cudaEventElapsedTime(&ms, e0, e1));
            if (ms < best) { best = ms; best_t = cand[q]; }
        }
        c.tpp = best_t;
        c.graph_dirty = 1;
        touch(c);
        if (tpp_out) tpp_out[r] = best_t;
        // the step expects the full forces of the current positions
        BCK(cudaMemsetAsync(c.acc, 0, ACC_COUNT * sizeof(long long), c.stream));
        enqueue_forces(c);
        BCK(cudaMemsetAsync(c.acc, 0, ACC_COUNT * sizeof(long long), c.stream));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->dirty = 1;
    return batch_status(b);
}

int smd_batch_run(smd_batch *b, int nsteps, double *device_ms) {
    if (!b || nsteps < 0) return SMD_ERR_ARG;
    BCK(cudaSetDevice(b->device));
    if (b->dirty || !b->graph) {
        const int r = batch_build(b);
        if (r) return r;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (device_ms) {
        BCK(cudaEventCreate(&e0));
        BCK(cudaEventCreate(&e1));
        BCK(cudaStreamSynchronize(b->stream));
        BCK(cudaEventRecord(e0, b->stream));
    }
    for (int s = 0; s < nsteps; s++) BCK(cudaGraphLaunch(b->graph, b->stream));
    if (device_ms) {
        BCK(cudaEventRecord(e1, b->stream));
        BCK(cudaEventSynchronize(e1));
        float ms = 0;
        BCK(cudaEventElapsedTime(&ms, e0, e1));
        *device_ms = ms;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    for (smd_ctx *x : b->reps) {
        x->c.steps_done += nsteps;
        if (nsteps > 0) touch(x->c);
    }
    return batch_status(b);
}

}  // extern "C"
