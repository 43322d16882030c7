// ref_minicell_shim.cpp -- TEST INFRASTRUCTURE.
//
// Lets the reference's own MiniCell (src/celeste/core/MiniCell.cpp), compiled unmodified
// from the reference tree, run on the CPU so that its cell assignment and cell-pair list
// can be compared bit for bit with the oracle (oracle/ogo.c) and the CUDA engine.
//
// MiniCell.cpp is compiled with -DF_CUDA -DF_ECP: in that configuration it allocates its
// coordinate array and obtains its host buffers through the cuda_hostalloc_* functions
// (MiniCell.cpp:7-35, 79-92).  This file supplies those functions as plain malloc/free,
// because the non-CUDA allocation path never allocates MiniCell::crd (it would crash).
// The expected number density argument sizes the per-column arrays
// (MiniCell.cpp:248-258) so that dense columns do not overflow them.
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <new>
#include <sstream>

#include "celeste/core/MiniCell.h"
#include "celeste/core/PBC.h"

extern "C" {

int cuda_hostalloc_atom_info(real_pw *&h_crd, int *&h_atomids, real_fc *&h_work, real_fc *&h_energy,
                             int max_n_atom_array) {
    size_t n = (size_t)max_n_atom_array + 64;
    h_crd    = (real_pw *)calloc(n * 3, sizeof(real_pw));
    h_atomids = (int *)calloc(n, sizeof(int));
    h_work   = (real_fc *)calloc(n * 3, sizeof(real_fc));
    h_energy = (real_fc *)calloc(4, sizeof(real_fc));
    return 0;
}
int cuda_hostalloc_cell_info(int *&h_idx_xy_head_cell, int n_columns) {
    h_idx_xy_head_cell = (int *)calloc((size_t)n_columns + 64, sizeof(int));
    return 0;
}
int cuda_hostfree_atom_info(real_pw *h_crd, int *h_atomids, real_fc *&h_work, real_fc *&h_energy) {
    free(h_crd);
    free(h_atomids);
    free(h_work);
    free(h_energy);
    return 0;
}
int cuda_hostfree_cell_info(int *h_idx_xy_head_cell) {
    free(h_idx_xy_head_cell);
    return 0;
}
int cuda_hostalloc_cellpair_info(CellPair *&h_cell_pairs, int *&h_idx_head_cell_pairs, int *&h_n_cells_z,
                                 int max_n_cell_pairs, int max_n_cells, int n_columns) {
    h_cell_pairs          = (CellPair *)calloc((size_t)max_n_cell_pairs + 64, sizeof(CellPair));
    h_idx_head_cell_pairs = (int *)calloc((size_t)max_n_cells + 64, sizeof(int));
    h_n_cells_z           = (int *)calloc((size_t)n_columns + 64, sizeof(int));
    return 0;
}
int cuda_hostfree_cellpair_info(CellPair *h_cell_pairs, int *h_idx_head_cell_pairs, int *&h_n_cells_z) {
    free(h_cell_pairs);
    free(h_idx_head_cell_pairs);
    free(h_n_cells_z);
    return 0;
}

// Runs SubBox::set_nsgrid's CPU sequence (SubBox.cpp:487-551) on one coordinate set and
// copies MiniCell's results out.  Returns 0, or -1 if a capacity is too small.
//   geom_i[8]: n_cells_x, n_cells_y, n_neighbors_x, n_neighbors_y, n_uni_z, n_columns, -, -
//   geom_f[4]: L_cell_x, L_cell_y, L_z_uni, -
int ogref_minicell(int n_atoms, const double *pbc_val, double nsgrid_cutoff, double density,
                   const double *crd_in, const int *nb15off_in, int max_nb15off,
                   int *geom_i, float *geom_f,
                   int cap_slots, int *n_cells_out, int *slot_atomid, double *slot_crd,
                   int cap_cols, int *col_head_cell,
                   int cap_pairs, int *n_pairs_out, int *idx_head, int *cell1, int *cell2, int *image,
                   unsigned int *mask /* 2 per pair */) {
    std::streambuf *saved = std::cout.rdbuf();
    std::ostringstream sink;
    std::cout.rdbuf(sink.rdbuf());

    PBC pbc;
    real val[12];
    for (int i = 0; i < 12; i++) val[i] = pbc_val[i];
    pbc.set_pbc(val);

    int *nb15off = new int[(size_t)n_atoms * max_nb15off];
    memcpy(nb15off, nb15off_in, sizeof(int) * (size_t)n_atoms * max_nb15off);
    real *crd = new real[(size_t)n_atoms * 3];
    int *ids  = new int[(size_t)n_atoms];
    for (int i = 0; i < n_atoms * 3; i++) crd[i] = crd_in[i];
    for (int i = 0; i < n_atoms; i++) ids[i] = i;

    // zero-filled storage: MiniCell's constructor leaves members (e.g. max_n_atoms_exbox)
    // uninitialised and set_max_n_atoms_region accumulates into it.
    void *mem    = calloc(1, sizeof(MiniCell));
    MiniCell *mc = new (mem) MiniCell();
    mc->set_grid_parameters(n_atoms, nsgrid_cutoff, &pbc, max_nb15off, nb15off, density);
    int nbox[3]    = {1, 1, 1};
    real box_l[3]  = {pbc.L[0], pbc.L[1], pbc.L[2]};
    mc->set_box_info(nbox, box_l);
    mc->set_max_n_atoms_region();
    mc->set_grid_xy();
    mc->alloc_variables();
    mc->set_crds_to_homebox(crd, ids, n_atoms);
    mc->set_atoms_into_grid_xy();
    mc->set_atomids_buf();
    mc->enumerate_cell_pairs();

    int rc = 0;
    const int *nxyz = mc->get_n_cells_xyz();
    const int *nn   = mc->get_n_neighbors_xyz();
    const real_pw *lc = mc->get_L_cell_xyz();
    geom_i[0] = nxyz[0];
    geom_i[1] = nxyz[1];
    geom_i[2] = nn[0];
    geom_i[3] = nn[1];
    geom_i[4] = mc->get_n_uni_z();
    geom_i[5] = mc->get_n_columns();
    geom_f[0] = lc[0];
    geom_f[1] = lc[1];
    geom_f[2] = mc->get_l_uni_z();

    int n_cells   = mc->get_n_cells();
    *n_cells_out  = n_cells;
    int n_slots   = n_cells * N_ATOM_CELL;
    int n_pairs   = mc->get_n_cell_pairs();
    *n_pairs_out  = n_pairs;
    int n_columns = mc->get_n_columns();
    if (n_slots > cap_slots || n_columns + 1 > cap_cols || n_pairs > cap_pairs) {
        rc = -1;
    } else {
        int *aids  = mc->get_atomids();
        real *gcrd = mc->get_crd();
        for (int s = 0; s < n_slots; s++) {
            slot_atomid[s] = aids[s];
            for (int d = 0; d < 3; d++) slot_crd[s * 3 + d] = gcrd[s * 3 + d];
        }
        int *head = mc->get_idx_xy_head_cell();
        for (int c = 0; c <= n_columns; c++) col_head_cell[c] = head[c];
        CellPair *cp = mc->get_cell_pairs();
        int *ih      = mc->get_idx_head_cell_pairs();
        for (int c = 0; c <= n_cells; c++) idx_head[c] = ih[c];
        for (int k = 0; k < n_pairs; k++) {
            cell1[k]        = cp[k].cell_id1;
            cell2[k]        = cp[k].cell_id2;
            image[k]        = cp[k].image;
            mask[2 * k]     = (unsigned int)cp[k].pair_mask[0];
            mask[2 * k + 1] = (unsigned int)cp[k].pair_mask[1];
        }
    }
    mc->~MiniCell();
    free(mem);
    delete[] crd;
    delete[] ids;
    // nb15off is owned by the caller of MiniCell in the reference (MmSystem); release it here.
    delete[] nb15off;
    std::cout.rdbuf(saved);
    return rc;
}

}  // extern "C"
