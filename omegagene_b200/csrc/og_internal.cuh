// og_internal.cuh -- device-side data layout shared by the engine's kernels.
//
// One engine holds S independent systems laid end to end in every array ("batch").
// Index spaces (all global across systems):
//   atom   -- original atom order, system s owns [atom_base, atom_base + n_atoms)
//   column -- MiniCell xy columns, system s owns [col_base, col_base + n_columns)
//   cell   -- 8-slot MiniCell cells, rebuilt on device; system s owns
//             [sys_cell_base[s], sys_cell_base[s+1])
//   slot   -- 8 * cell + k, grid order (MiniCell::atomids)
//   pair   -- cell pairs in CSR order over cell1
// Per-slot data are structure-of-arrays so that one warp reads 8-slot cells with
// coalesced 16-byte loads.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/omegagene_b200.h"

#define OG_CELL 8
#define OG_MAX_COLUMN_ATOMS 4096     // per-column sort capacity (shared memory)
#define OG_CELL_EXCL 32              // per-cell exclusion row: count + up to 31 (cell, bit) entries
#define OG_FIX_SCALE 4294967296.0    // 2^32: work (kcal/mol/A) -> int64 fixed point
#define OG_FIX_INV (1.0 / 4294967296.0)
#define OG_CHARGE_COEFF 332.06378    // CelesteObject.cpp:35
#define OG_FORCE_VEL 4.184e-4        // CelesteObject.cpp:36
#define OG_GAS_CONST 8.31451         // CelesteObject.cpp:37
#define OG_JOULE_CAL 4.184           // CelesteObject.cpp:38
#define OG_KINETIC_COEFF ((1e7 / (OG_JOULE_CAL * 1e3)) * 0.5)  // CelesteObject.cpp:39

// device error flags (bit set in d_counters[OG_CNT_FLAGS])
#define OG_FLAG_PAIR_CAPACITY 1
#define OG_FLAG_COLUMN_CAPACITY 2
#define OG_FLAG_BAD_COORD 4
#define OG_FLAG_SHAKE 8
#define OG_FLAG_THERMO 16
#define OG_FLAG_DISPLACEMENT 32      // an atom moved farther in one step than the list margin allows

// d_counters slots
#define OG_CNT_N_CELLS 0
#define OG_CNT_N_PAIRS 1
#define OG_CNT_FLAGS 2
#define OG_CNT_ACTIVE 3
#define OG_CNT_JL_STALE 4   // nonzero: the j lists must be rebuilt before the next pair launch
#define OG_CNT_JL_BUILDS 5  // j-list builds so far
#define OG_CNT_LIST_STALE 6 // displacement list policy: some atom moved half the list margin since the build
#define OG_CNT_LIST_BUILDS 7 // cell-pair list builds so far
#define OG_CNT_SIZE 8

// Per-system constants (read-only during a step).
struct SysDev {
    // box, PBC.h:21-27 (float) with double copies used by the FP64 integrator
    float Lf[3], lowerf[3], upperf[3], L_half_inv_f[3];
    double L[3], lower[3], upper[3];
    // MiniCell geometry (MiniCell.cpp:221-290)
    int nx, ny, n_columns, col_base;
    float L_cell[2];
    int n_nb[2], n_nb_cols;
    int n_uni_z, uni_base;
    float L_z_uni;
    float cutoff_pair2;          // nsgrid cutoff^2, float
    // atoms
    int atom_base, n_atoms;
    // pair interaction
    float cutoff2;               // interaction cutoff^2
    float zcore, bcoeff, fcoeff; // zero-dipole alpha=0 (ZeroMultipoleSum.cpp:150-202), float
    double cutoff;
    double max_step_disp2;       // squared displacement per step beyond which a system is faulted
    float list_trig2;            // displacement list policy: squared half margin, (nsgrid_cutoff - cutoff)^2 / 4
    int lj_base, n_types;
    int ljf_off;                 // the force-scaled copy (6 C6, 12 C12) of the LJ table starts here
    // integrator
    double dt;
    double temperature_coeff_thermo;  // Thermostat.cpp:13-16
    double temperature_coeff_dyn;     // DynamicsMode.cpp:67
    double tau_inv;
    double self_energy;
    int thermostat;
    int has_constraints;
    // V-McMD (ExtendedVMcMD, Extend.cpp:56-203): n_vs virtual states from vs_base of the state
    // table, n_vs = 0 when off.  vm_slot indexes the generator and log rings (-1: no transitions).
    int n_vs, vs_base, vm_slot, vs_trans_intvl, vs_lambda_intvl;
    long long first_step;             // step number of the engine's first step for this system
    // trajectory frames (DynamicsMode::sub_output): ring slot (-1: none), interval, group size,
    // and the offsets of the system's frame ring in the frame buffers
    int tr_slot, tr_interval, tr_n, tr_frames;
    long long tr_crd_base, tr_ene_base;
    double mcmd_k;                    // const_k = (GAS_CONST/JOULE_CAL) 1e-3 T
    // constraint / term ranges (global index spaces of their own arrays)
    int trio_base, n_trio, pair_base, n_pair;
    int excess_base, n_excess, bond_base, n_bonds, angle_base, n_angles;
    int tors_base, n_tors, impro_base, n_impro, nb14_base, n_nb14;
};

// One virtual state (VirtualState, Extend.cpp:20-55): lambda range, transition probabilities
// (trans_prob[0] down, trans_prob[1] up) and the d ln P / d lambda polynomial in raw powers.
struct VsDev {
    double lo, hi, p_down, p_up;
    double coef[8];
    int order;
};

// Electrostatics / nonbond model of a system other than zero-dipole alpha = 0 with plain LJ
// (ZeroMultipoleSum.cpp:108-466, ForceField.cpp:333-418).  FP32 coefficients for the pair
// kernel, as the reference's float members hold them; FP64 ones for the excluded-pair term.
struct EleDev {
    int mode, alpha0, hps, generic;
    float alpha, piewald, bcoeff, fcoeff, zcore, zqcore, zocore, zhcore;
    float zq2, zq4, zq22, zq44, zo2, zo4, zo6, zo22, zo44, zo66;
    float zh2, zh4, zh6, zh8, zh22, zh44, zh66, zh88;
    float dielectric_inv, debye_inv, hps_eps, zmcore;
    double d_alpha, d_piewald, d_bcoeff, d_fcoeff;
    double d_zq2, d_zq4, d_zq22, d_zq44, d_zo2, d_zo4, d_zo6, d_zo22, d_zo44, d_zo66;
    double d_zh2, d_zh4, d_zh6, d_zh8, d_zh22, d_zh44, d_zh66, d_zh88;
};

// per-system reduction slots in d_sys_acc (double)
#define OG_ACC_VDW 0
#define OG_ACC_ELE 1
#define OG_ACC_EXCESS 2
#define OG_ACC_BOND 3
#define OG_ACC_ANGLE 4
#define OG_ACC_KIN 5
#define OG_ACC_VIR 6     // 9 entries
#define OG_ACC_PAIRS 15  // interacting pair count of the last virial-mode evaluation
#define OG_ACC_TORSION 16
#define OG_ACC_IMPRO 17
#define OG_ACC_VDW14 18
#define OG_ACC_ELE14 19
#define OG_ACC_SIZE 20
// per-cell accumulator slots written by the pair kernel: vdw, ele, virial[9], pair count
#define OG_CELL_ACC 12

__device__ __forceinline__ unsigned int og_float_order(float f) {
    f = f + 0.0f;  // -0 -> +0 so that equal values give equal keys
    unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ void og_set_flag(int *counters, int flag) {
    atomicOr(&counters[OG_CNT_FLAGS], flag);
}

__device__ __forceinline__ long long og_to_fix(double w) {
    return __double2ll_rn(w * OG_FIX_SCALE);
}
