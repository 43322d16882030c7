/*
 * omegagene_celeste.h -- the reference's GPU interface, implemented on this engine.
 *
 * myPresto/omegagene's CELESTE_GPU build (-DF_CUDA) calls these extern "C" functions from its host
 * code: the declarations sit at the call sites, src/celeste/core/SubBox.cpp:5-78 and
 * src/celeste/core/MiniCell.cpp:7-35, and src/celeste/cuda/cuda_setup.cu defines them (file-scope
 * device globals, one system per process, sm_35 kernels).  libomegagene_celeste.so defines the
 * same functions with the same arguments on top of the og_* C ABI (omegagene_b200.h), so the
 * reference's program, compiled from its own sources with -DF_CUDA and linked against this library
 * instead of cuda_setup.cu, runs its MD with the cell-pair list and the pair LJ + zero-dipole
 * forces computed by this engine.  Everything else of the step stays where the reference keeps it:
 * MiniCell's host grid, the bonded and excluded-pair terms, the integrator, SHAKE and the
 * thermostat on the host.
 *
 * Roles (cuda_setup.cu line ranges of the functions replaced):
 *  - data: charges and types (cuda_memcpy_htod_atom_info, :115-123), LJ tables and exclusions
 *    (cuda_alloc_set_lj_params, :205-245), box (cuda_set_pbc, :138-147), cutoffs
 *    (cuda_set_constant, :193-204); the zero-dipole constants are recomputed by the engine from
 *    the cutoff in the same float arithmetic (cuda_zerodipole_constant, :148-156, is accepted
 *    and not needed);
 *  - per step: the grid-order float coordinates (cuda_memcpy_htod_crd + cuda_set_crd,
 *    :124-137, :427-434) go to the engine in atom order (og_put_state); cuda_pairwise_ljzd
 *    (:777-792) computes the pair forces over the engine's own cell-pair list, rebuilt from
 *    those coordinates after each cuda_enumerate_cell_pairs (:1095-1217), i.e. on the
 *    reference's nsgrid_update steps, and reused in between, as the reference reuses its list;
 *    cuda_memcpy_dtoh_work (:803-823) returns the work in the reference's grid order (its own
 *    atomids, cuda_memcpy_htod_atomids, :104-114) with the pair VDW and Ele energies;
 *  - host buffers: the cuda_hostalloc_* / cuda_hostfree_* pairs allocate host memory (the
 *    reference's are pinned; these are plain) that MiniCell and SubBox own.
 * Types follow the reference: real_pw is float, real_fc is double (CelesteObject.h:11-24).
 * Arguments passed by reference (T *&) are pointers in the C ABI.  On an engine error the
 * library prints og_last_error and exits the process, as the reference's HANDLE_ERROR does
 * (cuda_common.h:7-14); the og_* functions themselves never exit.
 * Not provided: the HPS / Debye-Hueckel GPU path (-DF_HPSCUDA, cuda_setup.cu:1230-1491) and the
 * host-enumerated list upload (-DF_ECP); their entry points return 1 and do nothing.
 */
#ifndef OMEGAGENE_CELESTE_H
#define OMEGAGENE_CELESTE_H

#ifdef __cplusplus
extern "C" {
int cuda_set_device(int device_id);
void cudaMemoryTest();
int cuda_alloc_atom_info(int max_n_atoms_exbox, int max_n_cells, int max_n_cell_pairs, int n_columns);
int cuda_free_atom_info();
int cuda_memcpy_htod_atom_info(float *&h_charge_orig, int *&h_atomtype_orig);
int cuda_set_cell_constant(const int in_n_cells, const int in_n_atoms_box, const int in_n_atom_array,
                           const int *in_n_cells_xyz, const int in_n_columns, const float *in_l_cell_xyz,
                           const int *in_n_neighbor_xyz);
int cuda_set_constant(float cutoff, float cutoff_pairlist, int n_atomtypes);
int cuda_alloc_set_lj_params(float *h_lj_6term, float *h_lj_12term, int n_lj_types, int *h_nb15off,
                             const int max_n_nb15off, const int max_n_atoms, const int max_n_atom_array);
int cuda_free_lj_params();
int cuda_memcpy_htod_atomids(int *&h_atomids, int *&h_idx_xy_head_cell);
int cuda_set_pbc(float *l, float *lb);
int cuda_memcpy_htod_crd(float *&h_crd);
int cuda_set_atominfo();
int cuda_set_crd();
int cuda_pairwise_ljzd(const bool flg_mod_15mask);
int cuda_memcpy_dtoh_work(double *&h_work, double *&h_energy, int n_atoms, int n_atom_array);
int cuda_pair_sync();
int cuda_thread_sync();
int cuda_zerodipole_constant(float zcore, float bcoeff, float fcoeff);
int cuda_hostfree_atom_type_charge(int *h_atom_type, float *h_charge);
int cuda_hostalloc_atom_type_charge(int *&h_atom_type, float *&h_charge, const int n_atoms_system);
int cuda_init_cellinfo(const int n_cells);
int cuda_enumerate_cell_pairs(int *&h_atomids, const int n_cells, const int n_neighbor_col,
                              const int *idx_atom_cell_xy);
int cuda_hostalloc_atom_info(float *&h_crd, int *&h_atomids, double *&h_work, double *&h_energy,
                             int max_n_atom_array);
int cuda_hostalloc_cell_info(int *&h_idx_xy_head_cell, int n_columns);
int cuda_hostfree_atom_info(float *h_crd, int *h_atomids, double *&h_work, double *&h_energy);
int cuda_hostfree_cell_info(int *h_idx_xy_head_cell);
/* not provided (return 1): */
int cuda_hps_constant(float epsiron);
int cuda_alloc_set_hps_params(float *h_hps_cutoff, float *h_hps_lambda, int n_lj_types);
int cuda_free_hps_params();
int cuda_debye_huckel_constant(float dielect, float temperature, float ionic_strength);
int cuda_pairwise_hps_dh(const bool flg_mod_15mask);
}
#endif

#endif
