/*
 * ogo -- CPU oracle for the omegagene per-step MD hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithms (myPresto/omegagene "celeste", CPU code path) used as the checker
 * for the CUDA engine in omegagene_b200/.  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / reference legs may load it.  The product never
 * calls into this library.
 *
 * Every function names the reference file:line it restates.  Float/double
 * semantics follow the reference's typedefs (CelesteObject.h:11-24):
 *   real = double, real_pw = float, real_fc = double, real_cst = double.
 * Build with -ffp-contract=off so that no multiply-add is fused.
 *
 * Parity pins (see tests/): the grid / cell-pair functions are compared bit for
 * bit with the reference's own MiniCell.cpp compiled from its sources
 * (oracle/build_ref.sh); the FP32 all-pairs energy path reproduces the
 * step-0 VDW and Ele of samples/ala3/log03_md.txt:127-135.
 */
#ifndef OGO_H
#define OGO_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OGO_N_ATOM_CELL 8
#define OGO_MAX_NB15OFF 32

/* PBC.h:21-27 -- all lengths are real_pw (float). */
typedef struct {
    float L[3], L_half[3], L_inv[3], L_half_inv[3], lower[3], upper[3];
} ogo_pbc;

/* MiniCell grid geometry (MiniCell.cpp:221-290, 1279-1303, 1327-1362). */
typedef struct {
    int   n_atoms;
    float cutoff_pair, cutoff_pair_half, cutoff_pair2;
    float exbox_l[3];
    float box_lower[3];
    int   n_cells_xy[2];
    float L_cell[2];
    int   n_columns;
    int   n_neighbors[2];
    int   n_uni_z;
    float L_z_uni;
} ogo_geom;

/* One MiniCell grid assignment (canonical slot order). */
typedef struct {
    int      n_cells;
    int      n_slots;          /* n_cells * 8 */
    int     *slot_atomid;      /* [n_slots]   original atom id, -1 for dummy */
    double  *slot_crd;         /* [n_slots*3] float-rounded coordinates (MiniCell::crd) */
    int     *atomids_rev;      /* [n_atoms]   atom id -> slot */
    int     *cell_column;      /* [n_cells]   column of each cell */
    int     *cell_z;           /* [n_cells]   z index of the cell in its column */
    int     *col_head_cell;    /* [n_columns+1] first cell of a column, -1 if empty; [n_columns] = n_cells */
    int     *col_n_atoms;      /* [n_columns] */
} ogo_grid;

/* Cell-pair list, CSR over cell1 (MiniCell.h:17-26). */
typedef struct {
    int       n_pairs;
    int      *idx_head;        /* [n_cells+1] */
    int      *cell1, *cell2, *image;
    uint64_t *mask;            /* bit a2*8+a1 set = pair skipped */
} ogo_cellpairs;

void ogo_pbc_init(ogo_pbc *p, const double val[12]);
int  ogo_geom_init(ogo_geom *g, const ogo_pbc *p, int n_atoms, double nsgrid_cutoff);

/* d[k] = minimum image of a[k] - b[k] (k < n, 3 doubles each): PBC::diff_crd_minim_image's two
 * truncating passes (PBC.cpp:70-84) and the guarded third one of the engine (ogo.c). */
void ogo_minim_image_d(const ogo_pbc *p, int n, const double *a, const double *b, double *d);

/* Wraps coordinates into the box like MmSystem::revise_crd_inbox (MmSystem.cpp:808-816). */
void ogo_revise_crd_inbox(const ogo_pbc *p, int n, double *crd);

/* reference_wrap = 1: the reference's column arithmetic, which wraps an in-box coordinate within
 * float rounding of the upper face into column 0 (MiniCell.cpp:329-335); 0: the engine's, which
 * keeps it in the last column, where its grid coordinate lies. */
int  ogo_grid_build(const ogo_geom *g, int n_atoms, const double *crd, int reference_wrap, ogo_grid *out);
void ogo_grid_free(ogo_grid *gr);
/* reference_faults = 1: the reference's uniform grid and bin scan, which register a cell whose
 * top lies within float rounding of the upper face in the next column (MiniCell.cpp:912-926) and
 * hide the cells of a neighbour column beyond a z gap of a bin's height (:1062-1076); 0: the
 * engine's list, which has neither fault. */
int  ogo_enumerate_cell_pairs(const ogo_geom *g, const ogo_pbc *p, const ogo_grid *gr,
                              const int *nb15off, int max_nb15off, int reference_faults, ogo_cellpairs *out);
void ogo_cellpairs_free(ogo_cellpairs *cp);

/* ZeroMultipoleSum::set_zms_params for alpha = 0 (ZeroMultipoleSum.cpp:150-202). */
void ogo_zd_constants(double cutoff, float *zcore, float *bcoeff, float *fcoeff);

/* FP32 pair path of the reference CPU build over the cell-pair list
 * (SubBox.cpp:956-1125, ForceField.cpp:333-418, ZeroMultipoleSum.cpp:309-332).
 * work_slot[n_slots*3] receives dE/dx per grid slot; ene[0]=VDW, ene[1]=Ele. */
void ogo_pair_cells_f32(const ogo_pbc *p, const ogo_grid *gr, const ogo_cellpairs *cp,
                        const float *charge, const int *atom_type, int n_types,
                        const float *lj6, const float *lj12, double cutoff,
                        float zcore, float bcoeff, float fcoeff,
                        double *work_slot, double ene[2]);

/* FP32 all-pairs path (SubBox.cpp:1127-1220), used with the ala3 known answer. */
void ogo_pair_allpairs_f32(const ogo_pbc *p, int n, const double *crd,
                           const float *charge, const int *atom_type, int n_types,
                           const float *lj6, const float *lj12, const int *nb15off, int max_nb15off,
                           double cutoff, float zcore, float bcoeff, float fcoeff,
                           double *work, double ene[2]);

/* FP64 oracle: every pair within cutoff, minimum image in double, LJ + ZD(alpha=0)
 * with double constants; virial W_ab = sum_pairs d_a f_b (d = x_i - x_j, f = force on i). */
void ogo_pair_allpairs_f64(const double L[3], int n, const double *crd,
                           const double *charge, const int *atom_type, int n_types,
                           const double *lj6, const double *lj12, const int *nb15off, int max_nb15off,
                           double cutoff, double *work, double ene[2], double vir[9]);

/* Same FP64 interaction evaluated over the cell-pair list (unrounded positions,
 * original atom order in and out).  O(N); equals the all-pairs result when the list
 * is complete. */
void ogo_pair_cells_f64(const double L[3], const ogo_grid *gr, const ogo_cellpairs *cp,
                        const double *crd, const double *charge, const int *atom_type, int n_types,
                        const double *lj6, const double *lj12, double cutoff,
                        double *work, double ene[2], double vir[9]);

/* Excluded-pair ZD correction (ForceField.cpp:420-437, SubBox.cpp:1347-1367). */
double ogo_excess_f32(const ogo_pbc *p, int n_excess, const int *excess_pairs, const double *crd,
                      const float *charge, float bcoeff, float fcoeff, double *work);
double ogo_excess_f64(const double L[3], int n_excess, const int *excess_pairs, const double *crd,
                      const double *charge, double cutoff, double *work, double vir[9]);

/* Self energy sum (ZeroMultipoleSum.cpp:43-106) with the float running sum. */
double ogo_self_energy(int n, int n_excess, const int *excess_pairs, const float *charge, float zcore);

/* ---- electrostatics and nonbond models other than zero-dipole alpha = 0 (ZeroMultipoleSum.cpp:
 * 108-466, ForceField.cpp:30-100,333-418).  Modes: --electrostatic zero-dipole / -quadrupole /
 * -octupole / -hexadecapole (alpha = --ele-alpha, 0 or > 0) and debye-huckel; HPS (--nonbond
 * hydrophobicity-scale-lj) scales the LJ term per type pair.  The formulas are the reference's,
 * including the places where they depart from the textbook forms (which the pin fixtures
 * confirm): the octupole alpha > 0 gradient uses the hexadecapole coefficients, and several
 * excess functions keep truncated or mismatched terms. */
#define OGO_ELE_ZD 0
#define OGO_ELE_ZQ 1
#define OGO_ELE_ZO 2
#define OGO_ELE_ZH 3
#define OGO_ELE_DH 4
typedef struct {
    int mode, alpha0;
    float alpha, cutoff, bcoeff, fcoeff, piewald, zmcore;
    float zcore, zqcore, zocore, zhcore;
    float zqcoeff2, zqcoeff4, zqcoeff22, zqcoeff44;
    float zocoeff2, zocoeff4, zocoeff6, zocoeff22, zocoeff44, zocoeff66;
    float zhcoeff2, zhcoeff4, zhcoeff6, zhcoeff8, zhcoeff22, zhcoeff44, zhcoeff66, zhcoeff88;
    float dielectric_inv, debye_length_inv;
} ogo_ele;
/* the same coefficients in double precision (FP64 oracle) */
typedef struct {
    int mode, alpha0;
    double alpha, cutoff, bcoeff, fcoeff, piewald, zmcore;
    double zcore, zqcore, zocore, zhcore;
    double zqcoeff2, zqcoeff4, zqcoeff22, zqcoeff44;
    double zocoeff2, zocoeff4, zocoeff6, zocoeff22, zocoeff44, zocoeff66;
    double zhcoeff2, zhcoeff4, zhcoeff6, zhcoeff8, zhcoeff22, zhcoeff44, zhcoeff66, zhcoeff88;
    double dielectric_inv, debye_length_inv;
} ogo_ele64;
/* HPS parameters: per type pair (n_types^2) cutoff and lambda; off when on == 0 */
typedef struct { int on; float eps; const float *cut, *lambda; } ogo_hps;
typedef struct { int on; double eps; const double *cut, *lambda; } ogo_hps64;

/* ZeroMultipoleSum constructor + set_zms_params (ZeroMultipoleSum.cpp:6-28,108-202) with the
 * reference's float members and double intermediates. */
void ogo_ele_init(ogo_ele *m, int mode, double alpha, double cutoff, double dh_dielectric,
                  double dh_ionic_strength, double dh_temperature);
void ogo_ele_init64(ogo_ele64 *m, int mode, double alpha, double cutoff, double dh_dielectric,
                    double dh_ionic_strength, double dh_temperature);
void ogo_pair_allpairs_f32_m(const ogo_pbc *p, int n, const double *crd, const float *charge, const int *atom_type,
                             int n_types, const float *lj6, const float *lj12, const int *nb15off, int max_nb15off,
                             double cutoff, const ogo_ele *m, const ogo_hps *h, double *work, double ene[2]);
void ogo_pair_cells_f64_m(const double L[3], const ogo_grid *gr, const ogo_cellpairs *cp, const double *crd,
                          const double *charge, const int *atom_type, int n_types, const double *lj6,
                          const double *lj12, double cutoff, const ogo_ele64 *m, const ogo_hps64 *h, double *work,
                          double ene[2], double vir[9]);
double ogo_excess_f32_m(const ogo_pbc *p, int n_excess, const int *excess_pairs, const double *crd,
                        const float *charge, const ogo_ele *m, double *work);
double ogo_excess_f64_m(const double L[3], int n_excess, const int *excess_pairs, const double *crd,
                        const double *charge, const ogo_ele64 *m, double *work, double vir[9]);
double ogo_self_energy_m(int n, int n_excess, const int *excess_pairs, const float *charge, const ogo_ele *m);

/* Excess pairs as MmSystem::set_excess_pairs builds them (MmSystem.cpp:700-736). */
int ogo_excess_pairs(int n, const int *nb15off, int max_nb15off, int *out_pairs /* [2*cap] */, int cap);

/* Bonds / angles (ForceField.cpp:108-177, SubBox.cpp:1229-1271). */
double ogo_bonds(const ogo_pbc *p, int n_bonds, const int *pairs, const double *k, const double *r0,
                 const double *crd, double *work);
double ogo_angles(const ogo_pbc *p, int n_angles, const int *triads, const double *k, const double *t0,
                  const double *crd, double *work);

/* ForceField::calc_torsion (ForceField.cpp:179-300) summed as SubBox::calc_energy_torsions /
 * calc_energy_impros (SubBox.cpp:1273-1320): E = ene (1 + cos(sym phi - phase)) / overlaps;
 * the same routine serves torsions and impropers.  Returns the energy, adds the work. */
double ogo_dihedrals(const ogo_pbc *p, int n, const int *quads, const double *ene, const int *overlaps,
                     const int *symmetry, const double *phase, const double *crd, double *work);
/* ForceField::calc_14pair (ForceField.cpp:302-331) summed as SubBox::calc_energy_14nb
 * (SubBox.cpp:1321-1345); charges and LJ terms are the reference's float values. */
void ogo_nb14(const ogo_pbc *p, int n, const int *pairs, const int *types, int n_types, const float *lj6,
              const float *lj12, const float *charge, const double *coeff_vdw, const double *coeff_ele,
              const double *crd, double *work, double *e_vdw, double *e_ele);

/* ---------------- integrator (DynamicsMode.cpp:468-560) ---------------- */
typedef struct {
    int     n;
    double  dt;
    /* state, original atom order */
    double *crd, *crd_prev, *vel, *vel_next, *work;
    const float *mass;       /* real_pw */
    float  *mass_inv;        /* real_pw */
    /* constraints (ConstraintShake.cpp) */
    int     n_pair, n_trio;
    const int    *pair_atoms;   /* [2*n_pair] */
    const double *pair_dist2;   /* squared */
    const int    *trio_atoms;   /* [3*n_trio] */
    const double *trio_dist2;   /* [3*n_trio] squared: d12, d23, d31 */
    int     n_quad;
    const int    *quad_atoms;   /* [4*n_quad] */
    const double *quad_dist2;   /* [6*n_quad] squared, pairs (0,1) (1,2) (2,0) (3,0) (2,3) (1,3) */
    int     shake_max_loops;
    double  shake_tol;
    /* COM cancel groups (COMMotion.cpp:30-55) */
    int     n_com_groups;
    const int *com_group_start;  /* [n_com_groups+1] into com_group_atoms */
    const int *com_group_atoms;
    const float *com_mass_inv;   /* real_pw mass_inv_groups */
    /* thermostat (Thermostat.cpp) */
    int     thermostat;          /* 0 none, 1 scaling */
    double  temperature;         /* target */
    double  temperature_coeff;   /* (2 JOULE_CAL 1e3)/(GAS_CONST d_free) KINETIC_COEFF */
    double  tau_inv;
    int     thermo_max_loops;
    double  thermo_tol;
    double *buf_crd;
} ogo_integ;

void   ogo_update_velocities(ogo_integ *s);                 /* SubBox.cpp:1427-1454 (incl. cpy_vel_prev) */
void   ogo_cancel_com(ogo_integ *s, double *v);             /* COMMotion.cpp:30-55 */
void   ogo_thermostat_scaling(ogo_integ *s);                /* Thermostat.cpp:57-84 */
void   ogo_update_coordinates(ogo_integ *s);                /* SubBox.cpp:1417-1420,1567-1580 */
void   ogo_shake(ogo_integ *s, const ogo_pbc *p);           /* ConstraintShake.cpp:10-149 */
void   ogo_set_velocity_from_crd(ogo_integ *s);             /* SubBox.cpp:1462-1481 */
int    ogo_thermostat_with_shake(ogo_integ *s, const ogo_pbc *p); /* Thermostat.cpp:86-170 */
void   ogo_revise_pbc(const ogo_pbc *p, int n, double *crd);      /* SubBox.cpp:1482-1502 */
void   ogo_move_grid(const ogo_grid *gr, int n, const double *crd, const double *crd_prev,
                     double *slot_crd);                              /* MiniCell.cpp:1312-1325 */
double ogo_kinetic(const ogo_integ *s, double *vel_just);          /* SubBox.cpp:1504-1516, DynamicsMode.cpp:358-372 */
/* V-McMD force scaling (Extend.cpp:114-117,178-203); returns the factor. */
double ogo_mcmd_scale(double lambda, double lam_low, double lam_high, int order, const double *coef,
                      double temperature, int n, double *work);
/* std::mt19937 as random::Random draws it (src/celeste/random/Random.cpp:20-28): st[0..623] the
 * words, st[624] the next position.  ogo_mt_seed = std::mt19937::seed(value). */
void     ogo_mt_seed(uint32_t *st, uint32_t seed);
uint32_t ogo_mt_next(uint32_t *st);
/* ExtendedVMcMD::set_current_vstate + trial_transition (Extend.cpp:144-177): the state after one
 * transition step; lam[2n] = low/high, prob[2n] = down/up of each state. */
int ogo_vmcmd_transition(int n_vs, const double *lam, const double *prob, int cur, double lambda, uint32_t *st);

#ifdef __cplusplus
}
#endif
#endif
