/* nnpe.h — C ABI of the B200 short-range force step (libnnpe.so).
 *
 * One context (nnpe_ctx) owns one periodic system resident in HBM: cell-sorted atoms, explicit
 * periodic images ("ghosts"), the Verlet neighbour list, tables, descriptors and accumulators.
 * Plain pointers and sizes only; host arrays are in atom-id order (the order of the
 * configuration file), which is how the reference's ENVIRON::atom_id indexes results.
 *
 * Every call returns 0 on success or an NNPE_E* code; nnpe_last_error() gives the message.
 * The reference ends the process on every such condition (END_PROGRAM, util.cpp:117-124); the
 * C++ adapter in nnpe.hpp maps a non-zero status back to that behaviour.
 *
 * The "replaces" notes cite the reference member each entry point stands in for
 * (paths within NNPEngine's src/).
 */
#ifndef NNPE_H
#define NNPE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nnpe_ctx nnpe_ctx;

enum {
  NNPE_OK = 0,
  NNPE_EARG = 1,       /* invalid argument or call order */
  NNPE_ECUDA = 2,      /* CUDA runtime error */
  NNPE_EOVERFLOW = 3,  /* a capacity was exceeded (list, ghosts, cell, stencil) */
  NNPE_EFILE = 4,      /* input file missing or malformed */
  NNPE_ERANGE = 5,     /* an atom left the cell grid */
  NNPE_ETIMEOUT = 6    /* a bounded device wait gave up */
};

/* Device error bits accumulated by kernels (nnpe_device_errors). */
enum {
  NNPE_DEV_LIST_OVERFLOW = 1,   /* "nei_list overflow", neighlist.cpp:327 */
  NNPE_DEV_GHOST_OVERFLOW = 2,  /* "ghost overflow", environ.cpp:440 */
  NNPE_DEV_CELL_RANGE = 4,      /* an atom or image outside the grid (CHECK_BINNING, environ.cpp:245-259) */
  NNPE_DEV_CELL_OVERFLOW = 8,   /* a cell holds more atoms than the in-cell sort supports */
  NNPE_DEV_NAN = 16,
  NNPE_DEV_TIMEOUT = 32,        /* a bounded wait on the tensor core gave up; the launch's results are void */
  NNPE_DEV_POISONED = 64        /* a kernel that gave up could not see its own asynchronous copies land:
                                   the context refuses further work (NNPE_ETIMEOUT) until nnpe_setup */
};

/* Per-log-step record of the step loop (run.cpp:376-392 prints the same quantities). */
typedef struct nnpe_thermo {
  int step;
  int nbuild;         /* NEIGHLIST::nbuild */
  double erg;         /* potential energy [kcal/mol] (FP64 reduction) */
  double virial;      /* sum of fpair*rsq [kcal/mol] */
  double ekin;        /* kinetic energy [kcal/mol] before the thermostat */
  double temperature; /* ekin/natom*ek_T [K] */
  double pressure;    /* (virial+2 ekin)/3 * ev_GPa / BL^3 [GPa] */
  double erg_nnp;     /* network part of erg */
  double erg_exp;     /* RMDF penalty of the last g(r) step (run.cpp:295, 386), 0 without RMDF */
} nnpe_thermo;

/* ---- context -------------------------------------------------------------------------- */
int nnpe_create(int device, nnpe_ctx** out);
void nnpe_destroy(nnpe_ctx* ctx);
const char* nnpe_last_error(const nnpe_ctx* ctx);
/* Raw device error bits since the last call to this function (then cleared). */
int nnpe_device_errors(nnpe_ctx* ctx, int* bits);
/* Device memory this context holds (bytes of its own allocations). */
int nnpe_device_bytes(const nnpe_ctx* ctx, int64_t* bytes);
/* Stream all work of this context is issued on (cudaStream_t as void*). */
void* nnpe_stream(nnpe_ctx* ctx);

/* ---- system (replaces ENVIRON::initialize, environ.cpp:22-141; MOLECULE::from_file,
 *      molecule.cpp:25-134) ------------------------------------------------------------- */
/* special: [nmoltype][nmax][nmax] special class per intra-molecule atom pair (0..3);
 * mol_rep: per molecule, the atom id of its representative (intra id 0). */
int nnpe_set_system(nnpe_ctx* ctx, int natom, int ntype, double bl, const int* typ, const float* mass,
                    const float* q, const float* x, const int* mol_id, const int* intra_id,
                    const int* atom_moltype, int nmoltype, int nmax, const int* special);
/* Parses the reference's initial-configuration file and its molecule files. */
int nnpe_load_system_file(nnpe_ctx* ctx, const char* init_file);
int nnpe_natom(const nnpe_ctx* ctx);
/* Atom types and molecule ids (atom-id order, int [natom]; NULL to skip) and the box edge. */
int nnpe_atom_info(const nnpe_ctx* ctx, int* typ, int* mol_id, double* bl);
int nnpe_npair(const nnpe_ctx* ctx);
/* Positions/velocities in atom-id order, float [natom*3]; replace the state in place. */
int nnpe_set_positions(nnpe_ctx* ctx, const float* x);
int nnpe_set_velocities(nnpe_ctx* ctx, const float* v);
/* ENVIRON::initV (environ.cpp:190-205): with probability frac per atom, Maxwell-Boltzmann
 * velocities at `temperature` [K]; the generator is seeded (the reference seeds from random_device). */
int nnpe_init_velocities(nnpe_ctx* ctx, double temperature, double frac, uint64_t seed);

/* ---- cutoffs, grid and stencils (replaces ENVIRON::init_grid environ.cpp:143-155,
 *      LOCAL::set_ghost_lim environ.h:142, NEIGHLIST::build_bin_list neighlist.cpp:35-168,
 *      NEIGHLIST ctor neighlist.cpp:13-33; wiring as run.cpp:72-82) ----------------------- */
/* neigh_cap: per-atom list capacity (NEIGH_SZ, run.h:2). nnp_cutoff > 0 adds the short
 * descriptor cutoff of a network term sharing the same list. */
int nnpe_setup(nnpe_ctx* ctx, double pair_cutoff, double skin, double gr_cutoff, int neigh_cap);
/* BL_MANAGER::setBL (run.cpp:688-712) with ENVIRON::set_bl (environ.h:105): a new cubic box length
 * for a set-up context. The grid keeps its cell length (half of cutoff + skin) and is re-derived
 * for the box, with its stencils and ghost limit; arrays that depend on the grid or on the image
 * count are reallocated. Positions are kept (they are in the caller's new box after
 * nnpe_set_positions or nnpe_force_step); the next evaluation rebuilds the list; the step counter
 * and the list-build count restart, as after nnpe_setup. A direct S(q) set-up holds the box it
 * was made for: call nnpe_sqd_setup again after a change. */
int nnpe_set_box(nnpe_ctx* ctx, double bl);

/* ---- LJTableCoulDSF (pair.h:30-54) ---------------------------------------------------- */
/* Tables [npair][nbin+1] of F(r)/r and U(r) at r=(i+.5)dr, dr=cutoff/nbin, last column 0
 * (replaces loadPotential, pair.cpp:197-263; the device copy is the `force/potential` pair). */
int nnpe_pair_set_table(nnpe_ctx* ctx, int nbin, const float* force, const float* potential);
int nnpe_pair_load_table(nnpe_ctx* ctx, int nbin, const char* potfile);
int nnpe_pair_get_table(nnpe_ctx* ctx, float* force, float* potential);
int nnpe_pair_enable(nnpe_ctx* ctx, int on);
/* on=1: fpair per pair in the reference's exact float sequence (IEEE sqrt/division, no FMA),
 * bit-identical to pair.cpp:334-357; on=0 (default): same cutoff test and table, rsqrt + FMA. */
int nnpe_pair_exact(nnpe_ctx* ctx, int on);

/* ---- bonded terms (BOND/ANGLE/DIHEDRAL, bond.h:6-21, angle.h:6-21, dihedral.h:4-17) ----
 * Terms in atom ids (as autoGenerate expands them, bond.cpp:66-86); coefficients in the
 * stored form of setParam: bond (b0, 2a, b, 2c), angle (cos t0, 2a, b, 2c), dihedral
 * (c0-c2, c1-3c3, 4c2, 12c3). */
/* setParam in the reference's float arithmetic: the stored forms above from raw parameters
 * (BOND::setParam bond.cpp:48-55, ANGLE::setParam angle.cpp:184-191 with theta0 in degrees,
 * DIHEDRAL::setParam dihedral.cpp:340-348). out: 4 floats. */
int nnpe_bond_coef(double b0, double ka, double kb, double kc, float* out);
int nnpe_angle_coef(double theta0, double ka, double kb, double kc, float* out);
int nnpe_dihedral_coef(double c0, double c1, double c2, double c3, float* out);
/* BOND/ANGLE/DIHEDRAL::autoGenerate (bond.cpp:66-103): the terms of every molecule read by
 * nnpe_load_system_file, with ntyp coefficient rows each in the stored form. */
int nnpe_bonded_autogen(nnpe_ctx* ctx, int nbtyp, const float* bcoef, int natyp, const float* acoef, int ndtyp,
                        const float* dcoef);
int nnpe_bonded_set(nnpe_ctx* ctx, int nbond, const int* bonds, int nbtyp, const float* bcoef, int nangle,
                    const int* angles, int natyp, const float* acoef, int ndih, const int* dihs, int ndtyp,
                    const float* dcoef);

/* ---- VERLET (verlet.h:4-22) and thermostat (run.cpp:348-373) --------------------------- */
/* fp64_state = 1: positions/velocities advanced in FP64 (default); 0: the reference's float
 * arithmetic, bit for bit. */
int nnpe_verlet_setup(nnpe_ctx* ctx, double dt, int fp64_state);
/* Number of steps the thermostat temperature ramp spans (total_steps of run.cpp:185). */
int nnpe_set_total_steps(nnpe_ctx* ctx, int total_steps);
/* thermostat: 0 none (NVE), 1 Andersen (re-draw `frac` of velocities, run.cpp:360-364),
 * 2 CSVR (run.cpp:365-372). Temperature ramps from t_start to t_end over the run. */
int nnpe_thermostat(nnpe_ctx* ctx, int kind, double t_start, double t_end, int interval, double frac,
                    uint64_t seed);

/* Single operations of the step for a caller that keeps the reference's own loop (nnpe.hpp):
 * VERLET::updateX with the given dt (the first call also clears the accelerations, run.cpp:220-221;
 * an atom that moved more than skin/2 since the last build marks the list invalid), and
 * VERLET::updateV with the kinetic energy (VERLET::computeKE, FP64 sum) when ekin != NULL. */
int nnpe_verlet_update_x(nnpe_ctx* ctx, double dt);
int nnpe_verlet_update_v(nnpe_ctx* ctx, double* ekin);

/* ---- the neighbour list (NEIGHLIST, neighlist.h:6-47) ---------------------------------- */
/* Rebuild: refold_and_tag, sort, generate_ghost, tidyup_ghost, update_ghost_pos<true>,
 * sort_ghost, update_ghost_and_info, build (run.cpp:249-276). */
int nnpe_list_build(nnpe_ctx* ctx);
/* NEIGHLIST::isvalid (neighlist.cpp:178-187), AND over all atoms. */
int nnpe_list_isvalid(nnpe_ctx* ctx, int* valid);
/* update_ghost_pos<false> (environ.cpp:488-522); with pruning on (nnpe_set_prune), also remakes
 * the pruned copy of the list when a rebuild or the displacement check asked for it. */
int nnpe_ghost_update(nnpe_ctx* ctx);
/* Sizes: natom, nghost, total list entries, nbuild. */
int nnpe_list_info(nnpe_ctx* ctx, int* nghost, int64_t* nentries, int* nbuild, int* num_gx);
/* Full list as records (atom id i, atom id j, image code, special class); image code
 * (sx+1)*9+(sy+1)*3+(sz+1) of the ghost shift, 13 for a real atom. cap = record capacity. */
int nnpe_list_get(nnpe_ctx* ctx, int64_t cap, int* rec, int64_t* n);
/* ENVIRON::verify_grid (environ.cpp:638-683), the cell sort's invariants: real atoms fill the
 * cells in order from index 0 and images from index natom, cell ranges are contiguous, and every
 * entry's stored cell is the cell of its position in the reference's float arithmetic. Where the
 * reference ends the program, these return NNPE_ERANGE. nnpe_verify_grid checks the context's
 * own sort (host copies; meaningful right after nnpe_list_build, as positions move between
 * builds). nnpe_verify_grid_arrays checks host arrays: cstart/cend/gcstart/gcend [num_gx^3],
 * cell [natom+nimage], pos4 [natom+nimage][4]; on a violation *bad is the cell or entry index
 * and *what its kind (1 bounds, 2 contiguity, 3 reversed range, 4 stored cell, 5 position's
 * cell). */
int nnpe_verify_grid(nnpe_ctx* ctx);
int nnpe_verify_grid_arrays(int natom, int nimage, int num_gx, float g_offset, float g_rdx, const int* cstart,
                            const int* cend, const int* gcstart, const int* gcend, const int* cell,
                            const float* pos4, int64_t* bad, int* what);
/* Dynamic pruning of the list (no counterpart in the reference, which evaluates every list entry;
 * the pairs that interact are the same). With delta > 0 (and below the skin) the pair and network
 * kernels read a copy of the list that keeps the entries within max(pair, network cutoff) + delta;
 * it is remade after every rebuild and whenever an atom has moved delta/2 since it was made, so it
 * holds every pair within the cutoffs. delta <= 0 or >= skin: off (the full list). Default 0.5 A.
 * The g(r) tally and nnpe_list_get always use the full list. */
int nnpe_set_prune(nnpe_ctx* ctx, double delta);
/* delta, whether the copy is in use, how many copies were made since nnpe_setup, and the entries
 * the current copy holds (any output may be null). */
int nnpe_prune_info(nnpe_ctx* ctx, double* delta, int* active, int* nprune, int64_t* nentries);

/* ---- forces (pair.cpp:289-419, bond/angle/dihedral compute, run.cpp:302-342) ------------
 * Clears the forces and evaluates pair + bonded (+ network when loaded) at the current
 * positions; erg/virial are FP64 device reductions (NULL to skip, i.e. ev=false). */
int nnpe_compute_forces(nnpe_ctx* ctx, int ev, double* erg, double* virial);
/* Force evaluation at host positions (atom-id order, float [natom*3]): the call a host-side
 * run loop makes in place of clear_vector/bond/angle/dihedral/pair.compute (run.cpp:302-342),
 * with the list check and rebuild of run.cpp:236-283 done on the device first. Writes the forces
 * to f_host (atom-id order); erg/virial (FP64) when non-NULL. */
int nnpe_force_step(nnpe_ctx* ctx, const float* x_host, float* f_host, double* erg, double* virial);
/* nnpe_force_step without any device allocation; no counterpart in the reference. Positions and
 * forces are staged in a static device array (3 MiB) instead of buffers allocated on first use,
 * for callers that cannot let the library allocate: a run loop whose process reserves the
 * device's memory for its own allocator, or one that cannot take the implicit inter-stream
 * synchronisation of an allocation. nnpe_setup resolves the array on the context's device (that
 * loads the module holding it and reserves the 3 MiB there, until the process exits), so this
 * call loads and reserves nothing; a device reset under a set-up context is not supported.
 * natom <= 131072, else NNPE_EARG. All contexts on a device share the array, so calls that
 * overlap in time race on it; serialise them. */
int nnpe_force_step_noalloc(nnpe_ctx* ctx, const float* x_host, float* f_host, double* erg, double* virial);
/* Forces (kind 0) or accelerations after the last step (kind 1), atom-id order [natom*3]. */
int nnpe_get_forces(nnpe_ctx* ctx, int kind, float* f);
int nnpe_get_positions(nnpe_ctx* ctx, float* x);
int nnpe_get_positions_f64(nnpe_ctx* ctx, double* x);
int nnpe_get_velocities(nnpe_ctx* ctx, float* v);
int nnpe_get_velocities_f64(nnpe_ctx* ctx, double* v);
/* Per-atom energies of the last ev evaluation, atom-id order (FP64). */
int nnpe_get_atom_energy(nnpe_ctx* ctx, double* e);

/* ---- the step loop (classical, run.cpp:192-394; nnp_run, run.cpp:1087-1354) -----------
 * Runs steps md_step=first..first+nsteps-1 of updateX, list check/rebuild, g(r) tally on
 * gr_interval, forces, updateV, thermostat; records one nnpe_thermo per log_interval into
 * log (capacity max_log, count in *nlog). The first call after setup performs the
 * reference's initial updateX with -dt (run.cpp:193-227). */
int nnpe_run(nnpe_ctx* ctx, int nsteps, int log_interval, nnpe_thermo* log, int max_log, int* nlog);
/* Same loop with all device work of each step captured once in a CUDA graph and replayed;
 * the rebuild decision stays on the device. */
int nnpe_run_graph(nnpe_ctx* ctx, int nsteps, int log_interval, nnpe_thermo* log, int max_log, int* nlog);

/* ---- network term (NNPOTENTIAL_TBL, pair_nnp.h:54-75) -----------------------------------
 * kind 0: the reference's tabulated NNP (20 Gaussian descriptors per special class from
 *   coef_w/coef_d/coef_r [npair][4][20], pair part from coef_p [npair][4][6]; tables generated as
 *   in the NNPOTENTIAL_TBL constructor, pair_nnp.cpp:521-590); e1/e2/scale/embw unused.
 * kind 1: radial embedding 1->e1->e2 (tanh) per neighbour species (e1=32), times the cutoff
 *   factor and `scale`, in descriptor slots s*e2+c (din=4*e2); coef_p may be NULL (no pair part).
 * fitw: per species A1[din][h1] c1[h1] A2[h1][h2] c2[h2] A3[h2] c3 (tanh hidden layers).
 * The network shares the pair list: cutoff <= pair_cutoff+skin. */
int nnpe_nnp_set(nnpe_ctx* ctx, int kind, double cutoff, int nbin, double scale, int e1, int e2, int h1, int h2,
                 const float* coef_p, const float* coef_w, const float* coef_d, const float* coef_r,
                 const float* embw, const float* fitw);
/* Reads the reference's NNP inputs: the paramfile (its first token names an NNPE model file:
 * text header, "end", float32 weights) and the reference-format weight file (bond/angle/dihedral
 * coefficients, coef_p, coef_w, coef_d, coef_r, pair_nnp.cpp:505-519), which, as in the reference,
 * also sets the bonded coefficients. */
int nnpe_nnp_load(nnpe_ctx* ctx, double cutoff, int nbin, const char* paramfile, const char* wtfile);
/* Switch the network term off/on (kept loaded). */
int nnpe_nnp_enable(nnpe_ctx* ctx, int on);
/* 0: FP32 on CUDA cores (the plain form); 1: BF16 operands on tcgen05 tensor cores, FP32 accumulate. */
int nnpe_nnp_precision(nnpe_ctx* ctx, int bf16);
/* Descriptor G, dE/dG (atom-id order, [natom][din]) and per-atom network energy of the last evaluation. */
int nnpe_nnp_get(nnpe_ctx* ctx, float* G, float* dEdG, double* e_atom);
int nnpe_nnp_info(nnpe_ctx* ctx, int* din, int* kind);
/* Pairs inside the network cutoff in the last evaluation (sum over atoms of the full list's count). */
int64_t nnpe_nnp_pairs(nnpe_ctx* ctx);

/* Grid sizes (CTAs) of the two tensor-core pair kernels (descriptor, force). The reference has no
 * counterpart: its network runs in TF on one thread. nnpe_nnp_autotune times candidate grids over
 * `reps` network evaluations of the current state (building the list if it is stale) and keeps the
 * fastest; with use_cache the choice is shared by contexts of the same device, species count and
 * half-octave of the atom count within the process. nnpe_nnp_grids sets them (0 = default: 4 and 2
 * CTAs per SM). The grid fixes how each CTA's pairs are cut into tiles: two runs with the same grid
 * give the same bits, different grids agree to FP32 rounding of the descriptor sums. */
int nnpe_nnp_autotune(nnpe_ctx* ctx, int reps, int use_cache, int* grid_desc, int* grid_force);
int nnpe_nnp_grids(nnpe_ctx* ctx, int grid_desc, int grid_force);
int nnpe_nnp_get_grids(nnpe_ctx* ctx, int* grid_desc, int* grid_force);

/* Self-test of the tcgen05 tile path on `device`: D[128][N] = bf16(A[128][K]) x bf16(B[N][K])^T,
 * FP32 accumulation in tensor memory (16 <= N <= 256, 16 <= K <= 128, multiples of 16).
 * mode 0: both operands K-major; 1: B MN-major; 2: A rows repeat with period 8 (one 8-row group
 * addressed with a zero stride); 3: modes 1 and 2 together. */
int nnpe_tc_selftest(int device, int mode, int N, int K, const float* A, const float* B, float* D);

/* ---- profiling ------------------------------------------------------------------------
 * Enqueue one kernel class without synchronising (for event timing): 0 pair force, 1 list
 * rebuild, 2 bonded, 3 network term, 4 Verlet, 5 cell-based g(r), 6 list-based g(r), 7 pair force
 * with the FP64 energy and virial (an energy step's pair pass). */
int nnpe_profile_enqueue(nnpe_ctx* ctx, int which);
/* Number of kernel launches in one plain MD step (the nodes of its CUDA graph). */
int nnpe_launches_per_step(nnpe_ctx* ctx);

/* ---- g(r) and S(q) (GR/SQ, grsq.h:8-38) -----------------------------------------------
 * GR(nbin_inner, gr_cutoff, pair_cutoff) bins (grsq.cpp:28-80); SQ(nq, qmax) (grsq.cpp:258-288). */
int nnpe_gr_setup(nnpe_ctx* ctx, int nbin_inner, int nq, double qmax, int gr_interval, int gr_interval_long);
/* Tally the current configuration (inner=1: list-based to the pair cutoff, grsq.cpp:94-149;
 * inner=0: cell-based to gr_cutoff, grsq.cpp:151-205) into fresh uint64 counts. */
int nnpe_gr_tally(nnpe_ctx* ctx, int inner);
int nnpe_gr_nbin(const nnpe_ctx* ctx, int inner);
/* counts [npair][nbin] (uint64, exact); gr [npair][nbin] = counts*norm-1 in FP64
 * (reduce_local grsq.cpp:207-219 with a double normaliser); sq [npair][nq] in FP64. */
int nnpe_gr_get(nnpe_ctx* ctx, int inner, uint64_t* counts, double* gr);
int nnpe_sq_compute(nnpe_ctx* ctx, int inner, double* sq, double* q);

/* ---- SQD (grsq.h:40-61): S(q) summed directly over reciprocal lattice vectors -------------
 * nnpe_sqd_setup is the SQD ctor (grsq.cpp:362-489): the half-space G set with |G| <= q_max, binned
 * on nq points, returns the vector count. nnpe_sqd_compute is SQD::compute (grsq.cpp:542-573) on the
 * current positions; nnpe_sqd_get returns the mean |G| per bin [nq], S(q) [nq][npair] (FP64) and
 * the vectors per bin [nq] (empty bins hold 0); nnpe_sqd_dump is SQD::dump (grsq.cpp:575-608). */
int nnpe_sqd_setup(nnpe_ctx* ctx, int nq, double qmax, int* ngv);
int nnpe_sqd_compute(nnpe_ctx* ctx);
int nnpe_sqd_get(nnpe_ctx* ctx, double* q, double* sq, int* count);
int nnpe_sqd_dump(nnpe_ctx* ctx, const char* fname, int append);

/* ---- RMDF (grsq.h:82-112): reverse-MD / FMIRL refinement of the pair table ---------------
 * RMDF ctor (grsq.cpp:899-1059) from arrays: n_sq targets, per q point (the SQ grid) S_exp, the
 * weight wt (multiplied by strength) and ntype scattering factors ff[n][q][t]. gamma = 1 is DA/RMD,
 * 0 <= gamma < 1 FMIRL. Refines LJTableCoulDSF's table when the pair term is on, else the network
 * term's pair tables (RMDF(..., nullptr, &nnp), run.cpp:1059). The table and g(r) grids must agree
 * ("RMDF mismatch", grsq.cpp:926-947). The table as it stands is kept as the base. Once set, every
 * g(r) step of nnpe_run/nnpe_run_graph runs compute_Qspace + compute_Rspace after S(q), and
 * compute_Potential on log steps when gamma != 1 (run.cpp:286-299). */
int nnpe_rmdf_set(nnpe_ctx* ctx, int n_sq, const double* sqex, const double* wt, const double* ff, double strength,
                  double gamma);
/* The same from the reference's target files: nq lines "q S_exp wt f_0 ... f_{ntype-1}". */
int nnpe_rmdf_load(nnpe_ctx* ctx, int n_sq, const char* const* files, double strength, double gamma);
/* RMDF::loadDeltaSQ (grsq.cpp:1419-1443); a missing file is ignored, as there. */
int nnpe_rmdf_load_delta(nnpe_ctx* ctx, const char* fname);
/* Parts of one update on the current S(q), as bits of `parts`: 1 compute_Qspace (erg_exp = the
 * penalty times natom/4, grsq.cpp:1117), 2 compute_Rspace, 4 compute_Potential (the _NNP variants
 * when the network's tables are refined). */
int nnpe_rmdf_step(nnpe_ctx* ctx, int parts, double* erg_exp);
/* Weighted S_n(q), deltaS_n(q) [n_sq][nq] and force_q [npair][nq] of the last update (NULL to skip). */
int nnpe_rmdf_get(nnpe_ctx* ctx, double* sq, double* deltasq, double* force_q);
/* RMDF::dumpSQ (grsq.cpp:1380-1416). */
int nnpe_rmdf_dump_sq(nnpe_ctx* ctx, const char* fname, int append);

/* ---- serving: a stream of independent MD replicas on one GPU ------------------------------
 * No counterpart in the reference, which holds one system per process (ENVIRON is a static
 * singleton, environ.h:20-123) and so runs such a stream as one run after another. A server owns a
 * worker thread that admits queued requests in arrival order as soon as a replica slot is free and
 * the request's device footprint fits the HBM budget, keeps a CUDA-graph launch of chunk_steps MD
 * steps in flight on every resident replica (replicas of different sizes overlap on the device; new
 * arrivals join while others run), and retires finished replicas. Each replica is a context as
 * above; its result does not depend on what else runs. */
typedef struct nnpe_server nnpe_server;

/* Force field and run settings shared by all replicas; arrays are copied by nnpe_server_create.
 * The pair table, bonded coefficients (stored forms) and network follow nnpe_pair_set_table,
 * nnpe_bonded_set and nnpe_nnp_set; force == NULL: no pair term; nnp_kind < 0: no network. */
typedef struct nnpe_serve_config {
  int device;
  int max_replicas;          /* resident replicas at most */
  int64_t hbm_budget;        /* device bytes the resident replicas may hold */
  int chunk_steps;           /* MD steps per launch; also the thermostat and log interval */
  double pair_cutoff, skin;
  int neigh_cap;
  double dt;
  int fp64_state;
  int thermostat;            /* 0 NVE, 1 Andersen (run.cpp:360-364) at the request's temperature */
  double thermo_frac;
  int ntype;
  int nbin;
  const float* force;        /* [npair][nbin+1] F(r)/r */
  const float* potential;    /* [npair][nbin+1] U(r) */
  int nbtyp;
  const float* bcoef;
  int natyp;
  const float* acoef;
  int ndtyp;
  const float* dcoef;
  int nnp_kind;
  double nnp_cutoff;
  int nnp_nbin;
  double nnp_scale;
  int e1, e2, h1, h2;
  const float *coef_p, *coef_w, *coef_d, *coef_r, *embw, *fitw;
  int nnp_bf16;
  int autotune;              /* tune the network kernels' grids per size class at admission (cached) */
} nnpe_serve_config;

/* One MD request: a system in the arrays of nnpe_set_system, initial velocities, bonded terms in
 * the form of nnpe_bonded_set, and nsteps MD steps (md_step 0..nsteps-1) at `temperature`
 * (Andersen when the server's thermostat is on; seed keys its random numbers). */
typedef struct nnpe_request {
  int natom;
  double bl;
  const int* typ;
  const float* mass;
  const float* q;
  const float* x;
  const float* v;
  const int* mol_id;
  const int* intra_id;
  const int* atom_moltype;
  int nmoltype, nmax;
  const int* special;
  int nbond;
  const int* bonds;
  int nangle;
  const int* angles;
  int ndih;
  const int* dihs;
  int nsteps;
  double temperature;
  uint64_t seed;
} nnpe_request;

typedef struct nnpe_request_stats {
  int64_t id;
  int natom, nsteps;
  int status;                    /* 0 queued, 1 resident, 2 done, < 0: failed with NNPE_E* code -status */
  double t_submit, t_admit, t_done;   /* seconds since the server was created */
  int64_t bytes;                 /* device bytes the replica held */
  double erg, ekin, temperature; /* last log record (first step of the last chunk) */
} nnpe_request_stats;

int nnpe_server_create(const nnpe_serve_config* cfg, nnpe_server** out);
/* Queues a copy of the request; returns at once with its id. */
int nnpe_server_submit(nnpe_server* srv, const nnpe_request* req, int64_t* id);
/* Blocks until request id is done (timeout_s < 0: no limit; NNPE_ETIMEOUT when it expires). */
int nnpe_server_wait(nnpe_server* srv, int64_t id, double timeout_s, nnpe_request_stats* st);
/* Final positions and velocities (atom-id order, float [natom*3]) of a finished request. */
int nnpe_server_result(nnpe_server* srv, int64_t id, float* x, float* v, nnpe_request_stats* st);
/* Blocks until every submitted request is done. */
int nnpe_server_drain(nnpe_server* srv, double timeout_s);
int nnpe_server_info(nnpe_server* srv, int64_t* done, int64_t* queued, int* resident, int64_t* bytes_in_use,
                     int64_t* peak_bytes, int* peak_resident);
/* Device bytes the admission test reserves for a request of natom atoms in a box of edge bl. */
int64_t nnpe_server_footprint(nnpe_server* srv, int natom, double bl);
const char* nnpe_server_error(nnpe_server* srv);
/* Stops the worker after the chunks in flight and frees every replica. */
void nnpe_server_destroy(nnpe_server* srv);

#ifdef __cplusplus
}
#endif
#endif /* NNPE_H */
