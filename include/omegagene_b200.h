/*
 * omegagene_b200.h -- C ABI of the B200 (sm_100a) engine for omegagene's per-step MD hot path:
 * MiniCell cell assignment + cell-pair list, the Lennard-Jones + zero-dipole pair kernel, and
 * the leapfrog integrator with SHAKE, velocity scaling and McMD force scaling.
 *
 * Plain C types only.  Every call returns an og_status and never exits the process
 * (the reference's HANDLE_ERROR exits, src/celeste/cuda/cuda_common.h:7-14).  State lives
 * behind an explicit handle; the reference keeps one system in file-scope device globals
 * (src/celeste/cuda/cuda_setup.h:32-134).  One engine holds one or more independent systems
 * ("batch"); every step kernel advances all of them in one launch.
 *
 * Units follow the reference: A, fs, amu, kcal/mol, e.  "work" is dE/dx (minus the force),
 * as in SubBox::work (src/celeste/core/SubBox.cpp:1445-1454).
 */
#ifndef OMEGAGENE_B200_H
#define OMEGAGENE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    OG_OK = 0,
    OG_ERR_INVALID = 1,   /* bad argument or unsupported input */
    OG_ERR_CUDA = 2,      /* CUDA runtime error (message in og_last_error) */
    OG_ERR_CAPACITY = 3,  /* a device buffer is too small (cell pairs, column size) */
    OG_ERR_STATE = 4,     /* call out of order (e.g. step before finalize) */
    OG_ERR_NOMEM = 5,     /* device allocation failed */
    OG_ERR_NOT_CONVERGED = 6, /* SHAKE / thermostat loop hit its iteration limit */
    OG_ERR_SYSTEM_FAULT = 7   /* og_step: some systems faulted, see og_get_system_faults */
} og_status;

typedef struct og_engine og_engine;

/* Thermostat kinds (CelesteObject.h THMSTT_*). */
#define OG_THERMOSTAT_NONE 0
#define OG_THERMOSTAT_SCALING 1

/* Energies reported per system (og_get_energies). */
#define OG_E_VDW 0
#define OG_E_ELE 1        /* pair + excluded-pair ("excess") ZD term + self energy */
#define OG_E_BOND 2
#define OG_E_ANGLE 3
#define OG_E_POTENTIAL 4
#define OG_E_KINETIC 5
#define OG_E_TEMPERATURE 6
#define OG_E_TOTAL 7
#define OG_E_ELE_EXCESS 8 /* excluded-pair ZD part of OG_E_ELE */
#define OG_E_ELE_SELF 9   /* constant self energy part of OG_E_ELE */
#define OG_E_MCMD_FACTOR 10
#define OG_E_TORSION 11
#define OG_E_IMPROPER 12
#define OG_E_VDW14 13     /* scaled 1-4 Lennard-Jones */
#define OG_E_ELE14 14     /* scaled 1-4 Coulomb */
#define OG_N_ENERGY 15    /* OG_E_POTENTIAL is the sum of VDW, ELE, BOND, ANGLE, TORSION, IMPROPER, VDW14, ELE14 */

/*
 * One system.  Arrays are host pointers in original atom order, copied by og_add_system.
 * Replaces the data the reference moves to the device through cuda_alloc_atom_info,
 * cuda_memcpy_htod_atom_info, cuda_alloc_set_lj_params, cuda_set_pbc,
 * cuda_zerodipole_constant and cuda_set_constant (src/celeste/cuda/cuda_setup.cu:42-300),
 * plus the host-side integrator inputs of SubBox / ConstraintShake / ThermostatScaling.
 */
typedef struct {
    int32_t n_atoms;
    double pbc_val[12];          /* .cls box block: L in [0],[4],[8]; box centre in [9..11] */
    const double *crd;           /* [3n] */
    const double *vel;           /* [3n] initial velocities (placed in vel_next as the reference does) */
    const double *charge;        /* [n] e */
    const double *mass;          /* [n] amu */
    const int32_t *atom_type;    /* [n] 0-based LJ types */
    int32_t n_lj_types;
    const double *lj6;           /* [n_lj_types^2]  C6 of E = C12/r^12 - C6/r^6 */
    const double *lj12;          /* [n_lj_types^2] */
    int32_t n_excl;              /* 1-5-off ("nb15off") pairs, each listed once */
    const int32_t *excl;         /* [2*n_excl] */
    int32_t n_shake_pair;        /* ConstraintShake pairs */
    const int32_t *shake_pair;   /* [2*n] */
    const double *shake_pair_dist;  /* [n] distance (not squared) */
    int32_t n_shake_trio;        /* ConstraintShake trios, e.g. (O, H1, H2) */
    const int32_t *shake_trio;   /* [3*n] */
    const double *shake_trio_dist;  /* [3*n] d12, d23, d31 (not squared) */
    int32_t n_bonds;
    const int32_t *bond;         /* [2*n] */
    const double *bond_k, *bond_r0;    /* E = k (r - r0)^2 */
    int32_t n_angles;
    const int32_t *angle;        /* [3*n] */
    const double *angle_k, *angle_t0;  /* E = k (theta - t0)^2, t0 in rad */
    int32_t n_com_groups;        /* COM translation cancelled per group (COMMotion.cpp:30-55) */
    const int32_t *com_group_start;  /* [n_com_groups+1] */
    const int32_t *com_group_atoms;
    /* run parameters (Config keys of the reference) */
    double cutoff;               /* --cutoff */
    double nsgrid_cutoff;        /* --nsgrid-cutoff */
    int32_t nsgrid_update_intvl; /* --nsgrid-update-intvl */
    double time_step;            /* --time-step (fs) */
    int32_t thermostat;          /* OG_THERMOSTAT_* (--thermostat) */
    double temperature;          /* --temperature */
    double temperature_init;     /* --temperature-init (<0: same as temperature) */
    int32_t heating_steps;       /* --heating-steps */
    double berendsen_tau;        /* --berendsen-tau (fs, after the reference's x1000) */
    int32_t const_max_loops;     /* --const-max-loops */
    double const_tolerance;      /* --const-tolerance */
    int32_t thermo_const_max_loops;    /* --thermo-const-max-loops */
    double thermo_const_tolerance;     /* --thermo-const-tolerance */
    /* V-McMD force scaling with one virtual state (Extend.cpp:178-203); order < 0 disables */
    int32_t mcmd_order;
    double mcmd_lambda_low, mcmd_lambda_high, mcmd_temperature;
    const double *mcmd_coef;     /* [order+1] */
    /* Step number of this system's first og_step (0 for a new run).  A run handed over between
     * engines (a serving loop re-forming its batch) passes the steps already done, a multiple of
     * nsgrid_update_intvl, so the heating schedule and the list-rebuild phase continue unchanged.
     * No counterpart in the reference, whose run always starts at step 0. */
    int64_t first_step;
    /* Dihedrals, E = ene (1 + cos(symmetry phi - phase)) / overlaps (ForceField::calc_torsion,
     * ForceField.cpp:179-300); torsions and impropers are reported separately. */
    int32_t n_torsions;
    const int32_t *torsion;          /* [4n] */
    const double *torsion_ene, *torsion_phase;       /* [n] kcal/mol, rad */
    const int32_t *torsion_overlaps, *torsion_symmetry; /* [n] */
    int32_t n_impros;
    const int32_t *impro;
    const double *impro_ene, *impro_phase;
    const int32_t *impro_overlaps, *impro_symmetry;
    /* 1-4 pairs (ForceField::calc_14pair, ForceField.cpp:302-331): scaled LJ and Coulomb without a
     * cutoff.  The factors are the ones the reference applies (its reader passes the .cls
     * record's two factors swapped, Read.cpp:438 against MmSystem.cpp:395-401). */
    int32_t n_nb14;
    const int32_t *nb14;             /* [2n] atoms */
    const int32_t *nb14_type;        /* [2n] 0-based LJ types */
    const double *nb14_coeff_vdw, *nb14_coeff_ele; /* [n] */
    /* SHAKE quads (ConstraintShake.cpp:151-276): centre + three partners; six distances in the
     * pair order (0,1) (1,2) (2,0) (3,0) (2,3) (1,3). */
    int32_t n_shake_quad;
    const int32_t *shake_quad;       /* [4n] */
    const double *shake_quad_dist;   /* [6n] A */
    /* Added to the degrees of freedom: 3 when the .cls holds a position-restraint section, as
     * Read.cpp:90-93 counts. */
    int32_t dof_extra;
    /* V-McMD with virtual-state transitions (ExtendedVMcMD, Extend.cpp:56-203; the .cls
     * "extended" section of Read::load_ls_vmcmd, Read.cpp:521-560).  n_vstates > 0 replaces the
     * one-state mcmd_* fields above (mcmd_temperature still gives const_k).  At every step s > 0
     * with s % vmcmd_trans_interval == 0 the system's state tries a move up, then down, with the
     * potential energy of that step as lambda (set_current_vstate / trial_transition,
     * Extend.cpp:144-177), and the forces are scaled with the polynomial of the state it is in
     * afterwards (scale_force, Extend.cpp:178-203).  Each trial draws from the system's own
     * std::mt19937 (random::Random, src/celeste/random/Random.cpp:20-28) seeded with vmcmd_seed:
     * the run's --random-seed (MmSystem::set_random, MmSystem.cpp:818-821; the seed stored in the
     * .cls section is not the one the reference draws with).  Steps count from the run's start,
     * first_step included. */
    int32_t n_vstates;
    int32_t vmcmd_trans_interval;     /* >= 1 */
    int32_t vmcmd_init_vs;            /* 0-based (the .cls holds it 1-based) */
    int32_t vmcmd_lambda_log_interval; /* --print-intvl-extended-lambda; 0: no lambda log */
    uint32_t vmcmd_seed;
    const int32_t *vs_order;          /* [n_vstates], each 0..7 */
    const double *vs_lambda;          /* [2 n_vstates]: low, high of each state's lambda range */
    const double *vs_prob;            /* [2 n_vstates]: down, up transition probability */
    const double *vs_coef;            /* polynomials, concatenated: [sum(order + 1)] */
    /* NULL for a new run; else [OG_MT_WORDS] generator words and position as og_get_vmcmd_state
     * returns them, so a run handed over between engines continues its random sequence. */
    const uint32_t *vmcmd_mt_state;
    /* Electrostatics and nonbond model (ForceField::set_config_parameters, ForceField.cpp:30-100;
     * ZeroMultipoleSum.cpp:6-28,108-466).  ele_mode OG_ELE_* (--electrostatic) with ele_alpha
     * (--ele-alpha) for the zero-multipole orders; Debye-Hueckel takes the three dh_* options
     * (--debye-huckel-dielectric / -ionic-strength [M] / -temperature [K]).  hps = 1
     * (--nonbond hydrophobicity-scale-lj) scales the LJ term per type pair: beyond the pair's
     * cutoff energy and force times lambda, inside it the energy plus (1 - lambda) hps_epsilon
     * (--hydrophobicity-scale-epsiron; ForceField.cpp:380-391); lj_hps_* are
     * [n_lj_types^2] tables as MmSystem::set_lj_pair_hps_param fills them.  All zero: the
     * zero-dipole alpha = 0 model with plain LJ. */
    int32_t ele_mode;
    double ele_alpha;
    double dh_dielectric, dh_ionic_strength, dh_temperature;
    int32_t hps;
    double hps_epsilon;
    const double *lj_hps_cutoff, *lj_hps_lambda;
} og_system_desc;

#define OG_ELE_ZD 0   /* zero-dipole */
#define OG_ELE_ZQ 1   /* zero-quadrupole */
#define OG_ELE_ZO 2   /* zero-octupole */
#define OG_ELE_ZH 3   /* zero-hexadecapole */
#define OG_ELE_DH 4   /* Debye-Hueckel */

/* std::mt19937 state: 624 words and the next position (624 = twist before the next draw). */
#define OG_MT_WORDS 625

/* Creates an engine on a CUDA device (cuda_set_device, cuda_setup.cu:1085-1093).  Debugging:
 * with OG_DEBUG_POISON=<byte> in the environment at creation, every device buffer the engine
 * allocates is first filled with that byte, so a kernel that reads memory nothing has written
 * yields results that depend on the byte (runs with two bytes must agree bit for bit). */
og_status og_create(int device, og_engine **out);
og_status og_destroy(og_engine *e);
/* Last error message of this engine ("" if none); valid until the next call. */
const char *og_last_error(const og_engine *e);

/* Adds a system (before og_finalize).  Its id is returned in sys_id (0, 1, ...). */
og_status og_add_system(og_engine *e, const og_system_desc *d, int32_t *sys_id);
/* Allocates device memory for every added system, uploads topology and state, builds the
 * cell grid and cell-pair list and computes the step-0 forces.  Replaces SubBox::set_nsgrid's
 * device part: gpu_device_setup, update_device_cell_info, cuda_enumerate_cell_pairs
 * (SubBox.cpp:487-551, 1683-1723; cuda_setup.cu:1095-1216). */
og_status og_finalize(og_engine *e);

/* Advances every system by n_steps of DynamicsModePresto::calc_in_each_step
 * (DynamicsMode.cpp:468-560), rebuilding the cell-pair list every nsgrid_update_intvl steps.
 * Replaces the per-step cuda_memcpy_htod_crd / cuda_set_crd / cuda_pairwise_ljzd /
 * cuda_memcpy_dtoh_work sequence (cuda_setup.cu:124-136, 777-823) and the host integrator. */
og_status og_step(og_engine *e, int32_t n_steps);

/* Rebuilds the cell grid and cell-pair list from the current coordinates and recomputes
 * forces and energies without advancing time (SubBox::nsgrid_update + SubBox::calc_energy). */
og_status og_compute_forces(og_engine *e);

/* Forces and energies at the current coordinates over the current cell-pair list, without
 * rebuilding it and without advancing time: the per-step force call of a caller that runs its own
 * integrator, as the reference's GPU path does (SubBox::calc_energy_pairwise_cuda ->
 * cuda_pairwise_ljzd, SubBox.cpp:906-955, cuda_setup.cu:777-801, with the list rebuilt only on
 * its nsgrid_update steps).  Coordinates come in through og_put_state; j lists that the move
 * made stale are rebuilt first.  Read the results with og_get_forces. */
og_status og_compute_forces_current(og_engine *e);
/* Before og_finalize: evaluate the pair Lennard-Jones + zero-dipole terms alone, without the
 * excluded-pair ZD term (and a caller gives no bonded terms): the share of the force field that
 * the reference computes on the GPU, its host computing the rest (SubBox::calc_energy,
 * SubBox.cpp:906-955).  OG_E_ELE is then the pair sum plus the self energy. */
og_status og_set_pair_only(og_engine *e, int32_t on);
/* Replaces a system's coordinates / velocities and marks the cell list for a rebuild at the
 * next step (synchronous). */
og_status og_set_state(og_engine *e, int32_t sys, const double *crd, const double *vel_next);
/* Continues the trajectory from host coordinates / velocities without re-enumerating cell
 * pairs (asynchronous, stream-ordered): the role of the reference's per-step
 * cuda_memcpy_htod_crd + cuda_set_crd (cuda_setup.cu:124-136, 380-402).  The grid copy moves
 * by the minimum-image displacement, as MiniCell::move_atom does (MiniCell.cpp:1312-1325).
 * Host buffers should be pinned for the copy to overlap. */
og_status og_put_state(og_engine *e, int32_t sys, const double *crd, const double *vel_next);
/* Stream-ordered device->host copies of state and energies (NULL pointers are skipped);
 * complete after og_synchronize.  The role of cuda_memcpy_dtoh_work (cuda_setup.cu:803-823). */
og_status og_get_state_async(og_engine *e, int32_t sys, double *crd, double *vel_next, double *energies);
/* Steps without the end-of-call synchronisation (see og_step); flags are read with og_get_flags.
 * Under the displacement list policy with graphs on (and no V-McMD system), the call's last step
 * (the one that computes energies) replays a captured one-step CUDA graph: its list rebuild is a
 * conditional node decided on the device, so the graph holds at any step.  The results equal
 * kernel-by-kernel steps bit for bit; the first such call captures the graph. */
og_status og_step_async(og_engine *e, int32_t n_steps);
og_status og_synchronize(og_engine *e);
og_status og_get_state(og_engine *e, int32_t sys, double *crd, double *vel_next);
/* work[3n] = dE/dx of the last force evaluation (pair + excess + bonded, before McMD scaling),
 * energies[OG_N_ENERGY], virial[9] = sum_pairs d_a f_b of the nonbonded (LJ + ZD) terms. */
og_status og_get_forces(og_engine *e, int32_t sys, double *work, double *energies, double *virial);
og_status og_get_energies(og_engine *e, int32_t sys, double *energies);
/* Interacting pairs (r < cutoff, not excluded) counted by the last og_compute_forces. */
og_status og_get_pair_count(og_engine *e, int32_t sys, int64_t *n_pairs);

/* Cell grid of the last list build (MiniCell's arrays in canonical order):
 * n_cells; slot_atomid[8*n_cells] (-1 dummy); col_head_cell[n_columns+1] (-1 empty column). */
og_status og_get_grid_info(og_engine *e, int32_t sys, int32_t *n_cells, int32_t *n_columns, int32_t *n_pairs);
og_status og_get_grid(og_engine *e, int32_t sys, int32_t *slot_atomid, double *slot_crd, int32_t *col_head_cell);
/* Cell-pair list in the reference's CSR order (MiniCell::enumerate_cell_pairs):
 * idx_head[n_cells+1], cell1/cell2/image[n_pairs], mask[n_pairs] (bit a2*8+a1 = skipped). */
og_status og_get_cell_pairs(og_engine *e, int32_t sys, int32_t *idx_head, int32_t *cell1, int32_t *cell2,
                            int32_t *image, uint64_t *mask);

/* Per-step energy trace: enables recording of the last `capacity` steps (0 disables). */
og_status og_set_trace(og_engine *e, int32_t capacity);
/* Copies up to max_steps recorded rows [steps][n_sys][OG_N_ENERGY]; returns the count in n_out. */
og_status og_get_trace(og_engine *e, double *out, int32_t max_steps, int32_t *n_out);

/* Launch statistics: kernels launched by the last og_step and device time of its pair kernel. */
og_status og_get_stats(og_engine *e, int64_t *kernel_launches, double *pair_kernel_ms, double *step_ms);
/* CUDA-event timing read with og_get_stats: on = 1 times every pair-kernel launch and the whole
 * og_step call (steps then launch kernel by kernel); on = 2 times only the whole og_step call
 * (graph replays stay on); 0 turns timing off. */
og_status og_set_timing(og_engine *e, int32_t on);
/* Device flags raised since the last og_step began: bit 8 = a SHAKE trio hit const_max_loops,
 * bit 16 = the thermostat loop hit thermo_const_max_loops (both non-fatal, as in the reference,
 * which prints a warning and continues: ConstraintShake.cpp:135-139, Thermostat.cpp:168). */
og_status og_get_flags(og_engine *e, int32_t *flags);
/* Pair-kernel variants: 0-2 = one warp per 8x8 cell pair at register budgets 100/80/64 per
 * thread; 3-4 = j-major (each lane one j atom against the 8 i atoms) at 100/80; 5-6 = j-major
 * with sm_100 packed FP32x2 arithmetic (two i atoms per instruction) at 128/80; 7-8 = packed
 * j-major fed by a per-warp queue of the j atoms within the cutoff of the i cell, at 128/80;
 * 9 = the same at 102 registers in blocks of 128 threads; 10 = packed j-major over j lists
 * culled once per list build (cutoff + 0.7 A around the i cell, rebuilt whenever an atom has
 * moved 0.35 A since), at 102 registers (engines with fewer than 2^24 atom slots).  An engine
 * holding a system with another electrostatics or nonbond model uses the generic forms of
 * variants 9 and 10 only (a fixed other variant means 9). */
#define OG_N_PAIR_VARIANTS 11
/* Not a tuned variant: the pair terms in FP64 throughout (positions, charges, C6/C12, every
 * operation) over the same cell-pair list, accumulated in the same fixed point.  A validation
 * mode for separating the production kernels' FP32 arithmetic from everything else of a
 * trajectory; several times slower; zero-dipole alpha = 0 with plain LJ only.  Chosen only with
 * og_set_tuning, never by the autotuner.  No counterpart in the reference, whose pair term is
 * FP32 (real_pw, CelesteObject.h:14). */
#define OG_PAIR_VARIANT_F64 11
/* Autotuner result: the pair-kernel variant in use and the best time of each variant on the
 * first list, in ms (variant_ms[OG_N_PAIR_VARIANTS]); for variant 10 the time is one step's
 * launch plus half a j-list build (the rate measured on water at 2 fs: one build per ~2.4 steps). */
og_status og_get_tuning(og_engine *e, int32_t *pair_variant, double *variant_ms);
/* Pair variant 10: j-list builds since og_finalize -- one at each cell-pair list build, plus one
 * whenever an atom has moved farther than the skin (0.35 A, or OG_JL_SKIN in the environment)
 * since the last.  0 for the other variants. */
og_status og_get_jlist_builds(og_engine *e, int64_t *n_builds);
/* Cell-pair list schedule, set before og_finalize (engine-wide).  OG_LIST_FIXED (default) is the
 * reference's: the list is rebuilt every nsgrid_update_intvl steps (DynamicsModePresto::
 * calc_in_each_step, DynamicsMode.cpp:480), and an atom that moves farther than the margin
 * (nsgrid_cutoff - cutoff) between rebuilds loses pairs, as in the reference.
 * OG_LIST_DISPLACEMENT rebuilds it before a step whenever an atom has moved farther than half the
 * margin since the last build (checked on the device every step; inside a graph replay the
 * build is a conditional node), so every pair within the cutoff is in the list: the list is
 * exact (with no margin, nsgrid_cutoff = cutoff, it is rebuilt every step).  In a batch the rebuild is engine-wide: one system's
 * moving atom rebuilds every system's list, so results are bitwise independent of the batch only
 * under OG_LIST_FIXED.  No counterpart in the reference. */
#define OG_LIST_FIXED 0
#define OG_LIST_DISPLACEMENT 1
og_status og_set_list_policy(og_engine *e, int32_t policy);
/* Cell-pair list builds since og_create (both policies; og_compute_forces builds one too). */
og_status og_get_list_builds(og_engine *e, int64_t *n_builds);
/* Fixes the pair-kernel variant (0..OG_N_PAIR_VARIANTS-1, or OG_PAIR_VARIANT_F64) before og_finalize and skips the autotuner, e.g. when a
 * serving loop re-creates engines for new batches; -1 restores autotuning.  No counterpart in
 * the reference, which has one pair kernel. */
og_status og_set_tuning(og_engine *e, int32_t pair_variant);
/* CUDA graphs (no counterpart in the reference, whose host loop launches every kernel each step):
 * og_step replays one captured graph per whole list interval -- the rebuild step and the
 * nsgrid_update_intvl-1 steps after it, the thermostat-with-SHAKE loop as a device-side WHILE
 * node -- when the step count covers it; other steps, and every step while og_set_timing(e, 1) is
 * on, launch kernel by kernel with identical results.  og_set_graphs(e, 0) turns graphs off
 * (default on).  og_get_graph_info reports whether graphs are on, how many replays ran and how
 * many kernel launches one replay stands for; `note` (may be NULL, 256 bytes) says why capture
 * turned graphs off, if it did. */
og_status og_set_graphs(og_engine *e, int32_t on);
/* After og_step returned OG_ERR_SYSTEM_FAULT: per system (faults[n_systems]) the bits of what went
 * wrong in it -- 4 = a non-finite or far out-of-box coordinate (the reference has no check and
 * carries on with NaNs), 32 = an atom moved farther in one step than the pair-list margin
 * (nsgrid_cutoff - cutoff, at least 1 A; the reference silently misses its pairs from then on),
 * 2 = more atoms in one MiniCell column than the engine sorts.  og_step
 * undid the whole call for every system (positions, velocities, step and trace counters are
 * those of the call's start); systems are independent, so a caller drops the faulted ones and
 * steps the rest in a new handle with the same results they would have had.  No counterpart in
 * the reference, which runs one system per process. */
og_status og_get_system_faults(og_engine *e, int32_t *faults);
/* Engines take device memory from one stream-ordered pool per device, which keeps what
 * og_destroy frees for the next engine of the process (a serving loop re-creates engines for
 * every new batch).  This returns the pool's unused reserve on `device` to the driver; it
 * synchronises that device first.  No counterpart in the reference, which allocates once per
 * run with cudaMalloc. */
og_status og_release_pool_memory(int32_t device);
og_status og_get_graph_info(og_engine *e, int32_t *enabled, int64_t *replays, int64_t *kernels_per_replay,
                            char *note);
/* Fixed-order FP64 sums of d_values[i*stride] over the segments [d_seg_base[s], d_seg_base[s+1])
 * of a device array, s < n_seg, into d_out[s] (device).  max_seg_len bounds every segment's
 * length.  The engine's own energy / kinetic-energy reduction (two levels: 4096-item chunks,
 * then chunks in order), so a segment's sum does not depend on the other segments.
 * Stream-ordered on cuda_stream (a cudaStream_t, NULL = default); its scratch is a
 * stream-ordered allocation released before return.  n_seg <= OG_SEGMENT_SUM_MAX_SEGMENTS
 * (one grid row per segment), else OG_ERR_CAPACITY.  A CUDA error already pending on the calling
 * thread is reported as OG_ERR_CUDA and left pending; nothing is launched then. */
#define OG_SEGMENT_SUM_MAX_SEGMENTS 65535
og_status og_segment_sum(const double *d_values, int32_t stride, const int32_t *d_seg_base, int32_t n_seg,
                         int32_t max_seg_len, double *d_out, void *cuda_stream);
/* og_segment_sum without any device allocation, for callers that cannot allocate at call time
 * (all free device memory already handed to another allocator's pool, or an allocation call not
 * acceptable on their path).  No counterpart in the reference.  Scratch is a fixed 512 KiB
 * array in device memory (n_seg <= OG_SEGMENT_SUM_MAX_SEGMENTS and
 * n_seg * ceil(max_seg_len / 4096) <= 65536, else OG_ERR_CAPACITY), held by every GPU that loads
 * the library until the process exits.  The first call on a device (with that device current)
 * looks up the array's device address; make that first call before any stream capture.  The
 * address is that of the device's primary context (the CUDA runtime's): call it from that
 * context only, and not after a cudaDeviceReset of the device.  All calls share the array:
 * calls that overlap on the GPU race. */
og_status og_segment_sum_noalloc(const double *d_values, int32_t stride, const int32_t *d_seg_base, int32_t n_seg,
                                 int32_t max_seg_len, double *d_out, void *cuda_stream);
/* Device memory the engine holds (bytes_held) and the most it has held at once (bytes_peak),
 * counting every buffer it allocated (the pair-list region grows when a list outgrows it).  A
 * serving loop sizes admission from these.  Either pointer may be NULL.  No counterpart in the
 * reference. */
og_status og_get_footprint(og_engine *e, int64_t *bytes_held, int64_t *bytes_peak);
/* Number of systems and atoms held. */
og_status og_get_sizes(og_engine *e, int32_t *n_systems, int64_t *n_atoms_total);

/* V-McMD state of a system after the last completed step: the 0-based virtual state
 * (ExtendedVMcMD::cur_vs) and, when mt_state is not NULL, the generator (OG_MT_WORDS words),
 * to hand the run to another engine through og_system_desc.vmcmd_init_vs / vmcmd_mt_state. */
og_status og_get_vmcmd_state(og_engine *e, int32_t sys, int32_t *cur_vs, uint32_t *mt_state);
/* Takes up to `max` of the oldest V-McMD log entries of a system that the caller has not taken
 * yet; *n receives how many were taken (with max = 0, how many there are).  Virtual-state log:
 * one entry per transition step, the step number and the 0-based state after the trial (the
 * reference writes "step<TAB>state+1" lines, WriteTTPVMcMDLog::write_ttpvMcMDLog,
 * Write.cpp:41-44, from apply_bias, Extend.cpp:128-131).  Lambda log: the step's potential
 * energy every vmcmd_lambda_log_interval steps (write_lambda, Extend.cpp:136, 252-255).  Entries
 * of a call undone by OG_ERR_SYSTEM_FAULT are dropped with it.  step / vs / lambda may be NULL
 * when max = 0. */
og_status og_take_vs_log(og_engine *e, int32_t sys, int64_t max, int64_t *step, int32_t *vs, int64_t *n);
og_status og_take_lambda_log(og_engine *e, int32_t sys, int64_t max, int64_t *step, double *lambda, int64_t *n);

/* Trajectory frames recorded on the device (DynamicsMode::sub_output, DynamicsMode.cpp:264-300;
 * --print-interval-coord / --group-o-coord).  Set before og_finalize: every `interval` steps
 * (0 = none) a frame of the group's atoms (n_group = 0: all atoms, local ids otherwise).  The
 * frame labelled step k (k > 0, k % interval == 0) holds what the reference writes there: the
 * coordinates at which step k-1's forces were computed (SubBox::crd_prev) rounded to FP32, as
 * WriteTrrPresto / WriteTrrGromacs store them, and step k-1's energies.  It is recorded at the
 * end of step k-1 inside og_step (graph replays included) and moved to the host before the
 * device ring wraps. */
og_status og_set_trajectory(og_engine *e, int32_t sys, int32_t interval, const int32_t *group_atoms,
                            int32_t n_group);
/* Takes up to `max` of the oldest frames not yet taken: steps[max], crd[max][n_group][3],
 * energies[max][OG_N_ENERGY] (may be NULL); *n = frames taken (with max = 0: frames waiting).
 * Frames of a call undone by OG_ERR_SYSTEM_FAULT are dropped with it. */
og_status og_take_frames(og_engine *e, int32_t sys, int32_t max, int64_t *step, float *crd, double *energies,
                         int32_t *n);

#ifdef __cplusplus
}
#endif
#endif
