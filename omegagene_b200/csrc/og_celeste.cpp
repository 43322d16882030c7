// og_celeste.cpp -- libomegagene_celeste.so: the reference's CELESTE_GPU entry points
// (include/omegagene_celeste.h) on top of this engine's og_* C ABI.
//
// The reference's host program keeps its MiniCell grid on the host and, per step, hands the GPU
// the grid-order float coordinates (MiniCell::get_crd_gpu, MiniCell.cpp:1239-1244) and the grid
// order itself (atomids: slot -> atom, -1 for padding); the GPU returns the pair work in the same
// grid order and the pair VDW / Ele energies (SubBox::calc_energy, SubBox.cpp:906-955).  Here one
// og_engine holds the system: its own on-device grid and cell-pair list, built from the same
// coordinates whenever the reference re-enumerates (cuda_enumerate_cell_pairs, i.e. its
// nsgrid_update steps) and reused in between, and only the pair terms evaluated (the host adds the
// bonded and excluded-pair terms, as with the reference's kernel).  The engine works in atom
// order; coordinates and work are mapped through the reference's atomids at the boundary.
//
// One system per process, as the reference's file-scope device state is.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/omegagene_b200.h"
#include "../../include/omegagene_celeste.h"

namespace {

struct Celeste {
    int device = 0;
    og_engine *eng = nullptr;
    int n_atoms = 0;  // atoms of the system (cuda_hostalloc_atom_type_charge)
    std::vector<double> charge;
    std::vector<int32_t> type;
    int n_lj_types = 0;
    std::vector<double> lj6, lj12;
    std::vector<int32_t> excl;  // each excluded pair once, i < j
    double L[3] = {0, 0, 0}, lower[3] = {0, 0, 0};
    double cutoff = 0, cutoff_pair = 0;
    int n_atom_array = 0;            // grid slots in use (cuda_set_cell_constant)
    std::vector<int> atomids;        // slot -> atom of the reference's grid
    std::vector<float> crd_grid;     // grid-order float coordinates of the last upload
    std::vector<double> crd;         // the same in atom order
    bool list_dirty = true;          // the reference re-enumerated since the last force call
    std::vector<double> work, ene;   // atom-order work and energies of the last force call
};

Celeste g;

void die(const char *what, og_status s) {
    std::fprintf(stderr, "omegagene_celeste: %s failed (og status %d): %s\n", what, (int)s,
                 g.eng ? og_last_error(g.eng) : "");
    std::exit(EXIT_FAILURE);
}

void check(og_status s, const char *what) {
    if (s != OG_OK) die(what, s);
}

// The engine's system from what the reference has handed over, at the first force call.
void create_engine() {
    og_system_desc d;
    std::memset(&d, 0, sizeof(d));
    d.n_atoms = g.n_atoms;
    d.pbc_val[0] = g.L[0];
    d.pbc_val[4] = g.L[1];
    d.pbc_val[8] = g.L[2];
    for (int q = 0; q < 3; q++) d.pbc_val[9 + q] = g.lower[q] + 0.5 * g.L[q];  // box centre (PBC.cpp:36)
    std::vector<double> vel(3 * (size_t)g.n_atoms, 0.0), mass((size_t)g.n_atoms, 1.0);
    d.crd = g.crd.data();
    d.vel = vel.data();
    d.charge = g.charge.data();
    d.mass = mass.data();  // unused: the reference integrates on the host
    d.atom_type = g.type.data();
    d.n_lj_types = g.n_lj_types;
    d.lj6 = g.lj6.data();
    d.lj12 = g.lj12.data();
    d.n_excl = (int32_t)(g.excl.size() / 2);
    d.excl = g.excl.data();
    d.cutoff = g.cutoff;
    d.nsgrid_cutoff = g.cutoff_pair;
    d.nsgrid_update_intvl = 1;
    d.time_step = 1.0;
    d.thermostat = OG_THERMOSTAT_NONE;
    d.temperature = 300.0;
    d.temperature_init = -1.0;
    d.const_max_loops = 1000;
    d.const_tolerance = 1e-7;
    d.thermo_const_max_loops = 100;
    d.thermo_const_tolerance = 1e-5;
    d.mcmd_order = -1;
    check(og_create(g.device, &g.eng), "og_create");
    check(og_set_pair_only(g.eng, 1), "og_set_pair_only");
    int32_t id = 0;
    check(og_add_system(g.eng, &d, &id), "og_add_system");
    check(og_finalize(g.eng), "og_finalize");  // builds the grid and list, computes the forces
}

}  // namespace

extern "C" {

int cuda_set_device(int device_id) {
    g.device = device_id;
    return 0;
}

void cudaMemoryTest() {}

int cuda_hostalloc_atom_type_charge(int *&h_atom_type, float *&h_charge, const int n_atoms_system) {
    g.n_atoms = n_atoms_system;
    h_atom_type = (int *)std::calloc((size_t)n_atoms_system + 1, sizeof(int));
    h_charge = (float *)std::calloc((size_t)n_atoms_system + 1, sizeof(float));
    return 0;
}

int cuda_hostfree_atom_type_charge(int *h_atom_type, float *h_charge) {
    std::free(h_atom_type);
    std::free(h_charge);
    return 0;
}

int cuda_hostalloc_atom_info(float *&h_crd, int *&h_atomids, double *&h_work, double *&h_energy,
                             int max_n_atom_array) {
    h_crd = (float *)std::calloc(3 * (size_t)max_n_atom_array, sizeof(float));
    h_atomids = (int *)std::calloc((size_t)max_n_atom_array, sizeof(int));
    h_work = (double *)std::calloc(3 * (size_t)max_n_atom_array, sizeof(double));
    h_energy = (double *)std::calloc(2, sizeof(double));
    return 0;
}

int cuda_hostfree_atom_info(float *h_crd, int *h_atomids, double *&h_work, double *&h_energy) {
    std::free(h_crd);
    std::free(h_atomids);
    std::free(h_work);
    std::free(h_energy);
    h_work = nullptr;
    h_energy = nullptr;
    return 0;
}

int cuda_hostalloc_cell_info(int *&h_idx_xy_head_cell, int n_columns) {
    h_idx_xy_head_cell = (int *)std::calloc((size_t)n_columns + 1, sizeof(int));
    return 0;
}

int cuda_hostfree_cell_info(int *h_idx_xy_head_cell) {
    std::free(h_idx_xy_head_cell);
    return 0;
}

int cuda_alloc_atom_info(int, int, int, int) { return 0; }  // the engine sizes its own buffers

int cuda_free_atom_info() {
    if (g.eng) og_destroy(g.eng);
    g.eng = nullptr;
    return 0;
}

int cuda_memcpy_htod_atom_info(float *&h_charge_orig, int *&h_atomtype_orig) {
    g.charge.assign((size_t)g.n_atoms, 0.0);
    g.type.assign((size_t)g.n_atoms, 0);
    for (int i = 0; i < g.n_atoms; i++) {
        g.charge[i] = (double)h_charge_orig[i];
        g.type[i] = h_atomtype_orig[i];
    }
    return 0;
}

int cuda_alloc_set_lj_params(float *h_lj_6term, float *h_lj_12term, int n_lj_types, int *h_nb15off,
                             const int max_n_nb15off, const int, const int) {
    g.n_lj_types = n_lj_types;
    g.lj6.assign(h_lj_6term, h_lj_6term + (size_t)n_lj_types * n_lj_types);
    g.lj12.assign(h_lj_12term, h_lj_12term + (size_t)n_lj_types * n_lj_types);
    g.excl.clear();
    for (int i = 0; i < g.n_atoms; i++)
        for (int k = 0; k < max_n_nb15off; k++) {
            const int j = h_nb15off[(size_t)i * max_n_nb15off + k];
            if (j < 0) break;
            if (i < j) {
                g.excl.push_back(i);
                g.excl.push_back(j);
            }
        }
    return 0;
}

int cuda_free_lj_params() { return 0; }

int cuda_set_pbc(float *l, float *lb) {
    for (int q = 0; q < 3; q++) {
        g.L[q] = (double)l[q];
        g.lower[q] = (double)lb[q];
    }
    return 0;
}

int cuda_set_constant(float cutoff, float cutoff_pairlist, int) {
    g.cutoff = (double)cutoff;
    g.cutoff_pair = (double)cutoff_pairlist;
    return 0;
}

int cuda_zerodipole_constant(float, float, float) { return 0; }

int cuda_set_cell_constant(const int, const int, const int in_n_atom_array, const int *, const int, const float *,
                           const int *) {
    g.n_atom_array = in_n_atom_array;
    return 0;
}

int cuda_memcpy_htod_atomids(int *&h_atomids, int *&) {
    g.atomids.assign(h_atomids, h_atomids + g.n_atom_array);
    return 0;
}

int cuda_set_atominfo() { return 0; }

int cuda_init_cellinfo(const int) { return 0; }

int cuda_memcpy_htod_crd(float *&h_crd) {
    g.crd_grid.assign(h_crd, h_crd + 3 * (size_t)g.n_atom_array);
    return 0;
}

// grid order -> atom order, as kernel_set_crd gathers it on the device (cuda_setup.cu:380-402)
int cuda_set_crd() {
    g.crd.assign(3 * (size_t)g.n_atoms, 0.0);
    for (int s = 0; s < g.n_atom_array; s++) {
        const int a = g.atomids[s];
        if (a < 0 || a >= g.n_atoms) continue;
        for (int q = 0; q < 3; q++) g.crd[3 * (size_t)a + q] = (double)g.crd_grid[3 * (size_t)s + q];
    }
    return 0;
}

int cuda_enumerate_cell_pairs(int *&, const int, const int, const int *) {
    g.list_dirty = true;  // the engine enumerates its own list from the coordinates of the next force call
    return 0;
}

int cuda_pairwise_ljzd(const bool) {
    if (!g.eng) {
        create_engine();
    } else if (g.list_dirty) {
        check(og_set_state(g.eng, 0, g.crd.data(), nullptr), "og_set_state");
        check(og_compute_forces(g.eng), "og_compute_forces");
    } else {
        check(og_put_state(g.eng, 0, g.crd.data(), nullptr), "og_put_state");
        check(og_compute_forces_current(g.eng), "og_compute_forces_current");
    }
    g.list_dirty = false;
    g.work.assign(3 * (size_t)g.n_atoms, 0.0);
    g.ene.assign(OG_N_ENERGY, 0.0);
    check(og_get_forces(g.eng, 0, g.work.data(), g.ene.data(), nullptr), "og_get_forces");
    return 0;
}

int cuda_pair_sync() { return 0; }  // the force call above completes before it returns
int cuda_thread_sync() { return 0; }

// atom-order work back to the reference's grid order; energy = pair VDW, pair Ele (no self or
// excluded-pair part: the host adds those, SubBox::calc_energy_ele_excess, DynamicsMode.cpp:444-458)
int cuda_memcpy_dtoh_work(double *&h_work, double *&h_energy, int, int n_atom_array) {
    for (int s = 0; s < n_atom_array; s++) {
        const int a = s < (int)g.atomids.size() ? g.atomids[s] : -1;
        for (int q = 0; q < 3; q++)
            h_work[3 * (size_t)s + q] = (a >= 0 && a < g.n_atoms) ? g.work[3 * (size_t)a + q] : 0.0;
    }
    h_energy[0] = g.ene[OG_E_VDW];
    h_energy[1] = g.ene[OG_E_ELE] - g.ene[OG_E_ELE_SELF] - g.ene[OG_E_ELE_EXCESS];
    return 0;
}

int cuda_hps_constant(float) { return 1; }
int cuda_alloc_set_hps_params(float *, float *, int) { return 1; }
int cuda_free_hps_params() { return 1; }
int cuda_debye_huckel_constant(float, float, float) { return 1; }
int cuda_pairwise_hps_dh(const bool) { return 1; }

}  // extern "C"
