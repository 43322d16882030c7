/*
 * ogo.c -- CPU oracle (TEST INFRASTRUCTURE, never the product path).
 * Plain-C restatement of the reference CPU algorithms; see ogo.h for scope.
 * Compile with: gcc -O2 -ffp-contract=off -fPIC -shared ogo.c -lm
 */
#include "ogo.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define CHARGE_COEFF 332.06378              /* CelesteObject.cpp:35 */
#define FORCE_VEL 4.184e-4                  /* CelesteObject.cpp:36 */
#define GAS_CONST 8.31451                   /* CelesteObject.cpp:37 */
#define JOULE_CAL 4.184                     /* CelesteObject.cpp:38 */
#define KINETIC_COEFF ((1e7 / (JOULE_CAL * 1e3)) * 0.5) /* CelesteObject.cpp:39 */

/* ------------------------------------------------------------------ PBC */

/* PBC::set_pbc (PBC.cpp:19-41): L, L_half, L_inv in float; lower bound from the
 * double box centre minus the float half length. */
void ogo_pbc_init(ogo_pbc *p, const double val[12]) {
    p->L[0] = (float)val[0];
    p->L[1] = (float)val[4];
    p->L[2] = (float)val[8];
    for (int i = 0; i < 3; i++) {
        p->L_half[i]     = (float)((double)p->L[i] * 0.5);
        p->L_inv[i]      = (float)(1.0 / (double)p->L[i]);
        p->L_half_inv[i] = (float)(1.0 / (double)p->L_half[i]);
        p->lower[i]      = (float)(val[9 + i] - (double)p->L_half[i]);
        p->upper[i]      = p->lower[i] + p->L[i];
    }
}

/* PBC::diff_crd_minim_image, double/double overload (PBC.cpp:70-84), plus one guarded pass.
 * The reference truncates d * L_half_inv to int twice.  Where float(2/L) * L rounds above 2,
 * a difference within L * (L * L_half_inv / 2 - 1) of +-L cycles +L -> -L through the two
 * truncations and comes back one box long instead of ~0 (a molecule split across opposite
 * faces with nearly equal x; the reference's SHAKE then diverges).  The third pass fires only
 * on such a result (|d| > 3L/4; every other two-pass result lies within L/2 of 0), so every
 * other output is the reference's bit for bit.  The engine applies the same pass. */
static void diff_minim_d(const ogo_pbc *p, double d[3], const double a[3], const double b[3]) {
    for (int i = 0; i < 3; i++) {
        d[i] = a[i] - b[i];
        d[i] = d[i] - (double)(p->L[i] * (float)(int)(d[i] * (double)p->L_half_inv[i]));
        d[i] = d[i] - (double)(p->L[i] * (float)(int)(d[i] * (double)p->L_half_inv[i]));
        if (fabs(d[i]) > 0.75 * (double)p->L[i]) d[i] = d[i] > 0.0 ? d[i] - (double)p->L[i] : d[i] + (double)p->L[i];
    }
}

/* The guarded minimum image above for n differences (tests). */
void ogo_minim_image_d(const ogo_pbc *p, int n, const double *a, const double *b, double *d) {
    for (int k = 0; k < n; k++) diff_minim_d(p, d + 3 * k, a + 3 * k, b + 3 * k);
}

/* PBC::diff_crd_minim_image, float/float overload (PBC.cpp:44-51), as the reference has it (no
 * guarded pass): it serves the all-pairs FP32 build, whose output the sample's log records. */
static void diff_minim_f(const ogo_pbc *p, float d[3], const float a[3], const float b[3]) {
    for (int i = 0; i < 3; i++) {
        d[i] = a[i] - b[i];
        d[i] = d[i] - p->L[i] * (float)(int)(d[i] * p->L_half_inv[i]);
        d[i] = d[i] - p->L[i] * (float)(int)(d[i] * p->L_half_inv[i]);
    }
}

void ogo_revise_crd_inbox(const ogo_pbc *p, int n, double *crd) {
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) {
            while (crd[i * 3 + d] < (double)p->lower[d]) crd[i * 3 + d] += (double)p->L[d];
            while (crd[i * 3 + d] >= (double)p->upper[d]) crd[i * 3 + d] -= (double)p->L[d];
        }
}

/* ------------------------------------------------------------ geometry */

/* MiniCell::set_grid_parameters (MiniCell.cpp:1279-1303), set_box_info (:1327-1362)
 * and set_grid_xy (:221-290), single box, no implicit-solvent density. */
int ogo_geom_init(ogo_geom *g, const ogo_pbc *p, int n_atoms, double nsgrid_cutoff) {
    memset(g, 0, sizeof(*g));
    g->n_atoms          = n_atoms;
    g->cutoff_pair      = (float)nsgrid_cutoff;
    g->cutoff_pair_half = (float)((double)g->cutoff_pair * 0.5);
    g->cutoff_pair2     = g->cutoff_pair * g->cutoff_pair;
    g->n_uni_z          = (int)(p->L[2] / g->cutoff_pair_half);
    if (g->n_uni_z < 1) return -1;
    g->L_z_uni = p->L[2] / (float)g->n_uni_z;
    for (int d = 0; d < 3; d++) {
        g->exbox_l[d]   = (float)(double)p->L[d];
        g->box_lower[d] = p->lower[d];
    }
    float volume = g->exbox_l[0] * g->exbox_l[1] * g->exbox_l[2];
    float w      = powf((float)((float)OGO_N_ATOM_CELL / ((float)n_atoms / volume)), (float)(1.0 / 3.0));
    if (w > g->cutoff_pair_half) w = g->cutoff_pair_half;
    for (int d = 0; d < 2; d++) {
        g->n_cells_xy[d] = (int)floorf(g->exbox_l[d] / w);
        if (g->n_cells_xy[d] < 1) return -1;
        g->L_cell[d]      = g->exbox_l[d] / (float)g->n_cells_xy[d];
        g->n_neighbors[d] = (int)ceilf(g->cutoff_pair / g->L_cell[d]);
        /* The reference indexes columns out of range when the neighbour reach exceeds
         * the column count; such boxes are rejected here and by the engine. */
        if (g->n_neighbors[d] > g->n_cells_xy[d]) return -2;
    }
    g->n_columns = g->n_cells_xy[0] * g->n_cells_xy[1];
    return 0;
}

/* ---------------------------------------------------------------- grid */

typedef struct { float z; int id; } zkey;
static int cmp_zkey(const void *a, const void *b) {
    const zkey *x = (const zkey *)a, *y = (const zkey *)b;
    if (x->z < y->z) return -1;
    if (x->z > y->z) return 1;
    return (x->id > y->id) - (x->id < y->id);
}

/* MiniCell::set_atoms_into_grid_xy (MiniCell.cpp:292-402) with reorder_atominfo_for_columns
 * (:404-501), set_dummy_atoms (:503-530), reorder_atominfo_in_columns + quick_sort_in_columns
 * (:531-613,636-691), set_idx_xy_head (:785-861), set_atomids_rev (:863-869).
 * The reference passes every coordinate through a float temporary while permuting atoms
 * into columns, then quicksorts each column on z.  Here each column is ordered by
 * (float z, atom id): identical to the reference wherever no two atoms of a column share
 * a float z, and a fixed tie order otherwise. */
int ogo_grid_build(const ogo_geom *g, int n_atoms, const double *crd, int reference_wrap, ogo_grid *out) {
    memset(out, 0, sizeof(*out));
    const int nc = g->n_columns;
    int *col_of  = (int *)malloc(sizeof(int) * (size_t)(n_atoms > 0 ? n_atoms : 1));
    out->col_n_atoms   = (int *)calloc((size_t)nc, sizeof(int));
    out->col_head_cell = (int *)malloc(sizeof(int) * (size_t)(nc + 1));
    for (int i = 0; i < n_atoms; i++) {
        int c[2];
        for (int d = 0; d < 2; d++) {
            float x = (float)(crd[i * 3 + d] - (double)g->box_lower[d]);
            if (!reference_wrap && x >= 0.0f && x <= g->exbox_l[d]) {
                /* an in-box coordinate stays in the column that holds it: within a few
                 * microangstroms of the upper face, x or x / L_cell rounds up to the box length or
                 * the column count, which the reference wraps to column 0 (MiniCell.cpp:329-335,
                 * :1251-1259), one box length from the coordinate the grid keeps for the atom */
                int ci = (int)floorf(x / g->L_cell[d]);
                c[d] = ci < g->n_cells_xy[d] ? ci : g->n_cells_xy[d] - 1;
                continue;
            }
            while (x < 0.0f) x += g->exbox_l[d];
            while (x >= g->exbox_l[d]) x -= g->exbox_l[d];
            c[d] = (int)floorf(x / g->L_cell[d]);
        }
        /* MiniCell::get_column_id_from_crd (:1251-1259) */
        while (c[0] < 0) c[0] += g->n_cells_xy[0];
        while (c[0] >= g->n_cells_xy[0]) c[0] -= g->n_cells_xy[0];
        while (c[1] < 0) c[1] += g->n_cells_xy[1];
        while (c[1] >= g->n_cells_xy[1]) c[1] -= g->n_cells_xy[1];
        col_of[i] = c[0] + c[1] * g->n_cells_xy[0];
        out->col_n_atoms[col_of[i]]++;
    }
    int n_cells = 0;
    for (int col = 0; col < nc; col++) {
        int ncz = (out->col_n_atoms[col] + OGO_N_ATOM_CELL - 1) / OGO_N_ATOM_CELL;
        out->col_head_cell[col] = out->col_n_atoms[col] == 0 ? -1 : n_cells;
        n_cells += ncz;
    }
    out->col_head_cell[nc] = n_cells;
    out->n_cells     = n_cells;
    out->n_slots     = n_cells * OGO_N_ATOM_CELL;
    out->slot_atomid = (int *)malloc(sizeof(int) * (size_t)(out->n_slots + 1));
    out->slot_crd    = (double *)malloc(sizeof(double) * 3 * (size_t)(out->n_slots + 1));
    out->atomids_rev = (int *)malloc(sizeof(int) * (size_t)(n_atoms + 1));
    out->cell_column = (int *)malloc(sizeof(int) * (size_t)(n_cells + 1));
    out->cell_z      = (int *)malloc(sizeof(int) * (size_t)(n_cells + 1));
    /* bucket atoms per column */
    int *start = (int *)malloc(sizeof(int) * (size_t)(nc + 1));
    start[0] = 0;
    for (int col = 0; col < nc; col++) start[col + 1] = start[col] + out->col_n_atoms[col];
    int  *fill = (int *)calloc((size_t)nc, sizeof(int));
    zkey *keys = (zkey *)malloc(sizeof(zkey) * (size_t)(n_atoms > 0 ? n_atoms : 1));
    for (int i = 0; i < n_atoms; i++) {
        int col = col_of[i];
        keys[start[col] + fill[col]].z  = (float)crd[i * 3 + 2];
        keys[start[col] + fill[col]].id = i;
        fill[col]++;
    }
    for (int col = 0; col < nc; col++) {
        int na = out->col_n_atoms[col];
        if (na == 0) continue;
        zkey *k = keys + start[col];
        qsort(k, (size_t)na, sizeof(zkey), cmp_zkey);
        int head = out->col_head_cell[col];
        int ncz  = (na + OGO_N_ATOM_CELL - 1) / OGO_N_ATOM_CELL;
        for (int cz = 0; cz < ncz; cz++) {
            out->cell_column[head + cz] = col;
            out->cell_z[head + cz]      = cz;
        }
        int slot0 = head * OGO_N_ATOM_CELL;
        for (int s = 0; s < ncz * OGO_N_ATOM_CELL; s++) {
            int src = s < na ? k[s].id : k[na - 1].id;
            int sl  = slot0 + s;
            out->slot_atomid[sl] = s < na ? src : -1;
            for (int d = 0; d < 3; d++) out->slot_crd[sl * 3 + d] = (double)(float)crd[src * 3 + d];
            if (s < na) out->atomids_rev[src] = sl;
        }
    }
    free(col_of);
    free(start);
    free(fill);
    free(keys);
    return 0;
}

void ogo_grid_free(ogo_grid *gr) {
    free(gr->slot_atomid);
    free(gr->slot_crd);
    free(gr->atomids_rev);
    free(gr->cell_column);
    free(gr->cell_z);
    free(gr->col_head_cell);
    free(gr->col_n_atoms);
    memset(gr, 0, sizeof(*gr));
}

/* --------------------------------------------------------- cell pairs */

/* MiniCell::check_valid_pair (MiniCell.cpp:1152-1162) */
static int valid_pair(int c1, int c2) {
    int o1 = c1 % 2 != 0, o2 = c2 % 2 != 0;
    if (o1) {
        if ((c2 < c1 && !o2) || (c2 > c1 && o2)) return 0;
    } else {
        if ((c2 < c1 && o2) || (c2 > c1 && !o2)) return 0;
    }
    return 1;
}

/* MiniCell::set_cell_pair_bitmask (MiniCell.cpp:1204-1237) */
static uint64_t pair_mask(const ogo_grid *gr, int c1, int c2, const int *nb15off, int max_nb15off) {
    uint64_t m = 0;
    for (int i1 = 0; i1 < OGO_N_ATOM_CELL; i1++) {
        int a1   = c1 * OGO_N_ATOM_CELL + i1;
        int id1  = gr->slot_atomid[a1];
        for (int i2 = 0; i2 < OGO_N_ATOM_CELL; i2++) {
            int a2  = c2 * OGO_N_ATOM_CELL + i2;
            int id2 = gr->slot_atomid[a2];
            int f   = 0;
            if (id1 == -1) f = 1;
            else if (id2 == -1) f = 1;
            else if (c1 == c2 && a1 >= a2) f = 1;
            else {
                const int *ex = nb15off + (size_t)id1 * max_nb15off;
                for (int k = 0; k < max_nb15off && ex[k] != -1; k++)
                    if (ex[k] == id2) { f = 1; break; }
            }
            if (f) m |= (uint64_t)1 << (i2 * OGO_N_ATOM_CELL + i1);
        }
    }
    return m;
}

/* MiniCell::set_uniform_grid (MiniCell.cpp:896-932) and enumerate_cell_pairs (:934-1150),
 * add_cell_pair (:1163-1203).  Loop order and float arithmetic are those of the
 * reference, so the list comes out in the reference's order. */
int ogo_enumerate_cell_pairs(const ogo_geom *g, const ogo_pbc *p, const ogo_grid *gr,
                             const int *nb15off, int max_nb15off, int reference_faults, ogo_cellpairs *out) {
    memset(out, 0, sizeof(*out));
    const int nx = g->n_cells_xy[0], ny = g->n_cells_xy[1], nuz = g->n_uni_z;
    const int n_uni = g->n_columns * nuz;
    const int n_cells = gr->n_cells;
    int *uni_lo = (int *)malloc(sizeof(int) * (size_t)n_uni);
    int *uni_hi = (int *)malloc(sizeof(int) * (size_t)n_uni);
    int *cu     = (int *)malloc(sizeof(int) * 2 * (size_t)(n_cells + 1));
    for (int i = 0; i < n_uni; i++) uni_lo[i] = uni_hi[i] = -1;
    for (int c = 0; c < n_cells; c++) {
        int   col  = gr->cell_column[c];
        int   cx   = col % nx, cy = col / nx, cz = gr->cell_z[c];
        float zmin = (float)gr->slot_crd[(c * OGO_N_ATOM_CELL) * 3 + 2] - p->lower[2];
        float zmax = (float)gr->slot_crd[(c * OGO_N_ATOM_CELL + OGO_N_ATOM_CELL - 1) * 3 + 2] - p->lower[2];
        int   umin = (int)(zmin / g->L_z_uni);
        int   umax = (int)(zmax / g->L_z_uni);
        if (!reference_faults) {
            /* a top within float rounding of the upper face divides out to bin nuz, which the
             * reference registers in the next column's bin 0 (MiniCell.cpp:912-926): its own
             * column never finds the cell.  It belongs to bin nuz - 1. */
            if (umin > nuz - 1) umin = nuz - 1;
            if (umax > nuz - 1) umax = nuz - 1;
        }
        cu[c * 2] = umin;
        cu[c * 2 + 1] = umax;
        for (int z = umin; z <= umax; z++) {
            int u = cx * nuz + cy * (nuz * nx) + z;
            if (u < 0 || u >= n_uni) continue; /* out of the reference's array */
            if (uni_lo[u] < 0 || cz < uni_lo[u]) uni_lo[u] = cz;
            if (cz > uni_hi[u]) uni_hi[u] = cz;
        }
    }
    int cap = n_cells * 16 + 16, n = 0;
    out->idx_head = (int *)malloc(sizeof(int) * (size_t)(n_cells + 1));
    out->cell1    = (int *)malloc(sizeof(int) * (size_t)cap);
    out->cell2    = (int *)malloc(sizeof(int) * (size_t)cap);
    out->image    = (int *)malloc(sizeof(int) * (size_t)cap);
    out->mask     = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)cap);
    for (int c1 = 0; c1 < n_cells; c1++) {
        int   col1 = gr->cell_column[c1];
        int   x1 = col1 % nx, y1 = col1 / nx;
        out->idx_head[c1] = n;
        float z1b = (float)gr->slot_crd[(c1 * OGO_N_ATOM_CELL) * 3 + 2];
        float z1t = (float)gr->slot_crd[(c1 * OGO_N_ATOM_CELL + OGO_N_ATOM_CELL - 1) * 3 + 2];
        for (int dcx = -g->n_neighbors[0]; dcx <= g->n_neighbors[0]; dcx++) {
            int rx = x1 + dcx, ix = 0, x2 = rx;
            if (rx < 0) { ix = -1; x2 = nx + rx; }
            else if (rx >= nx) { ix = 1; x2 = rx - nx; }
            float dx0;
            if (dcx > 0) dx0 = (float)(dcx - 1) * g->L_cell[0];
            else if (dcx < 0) dx0 = (float)(dcx + 1) * g->L_cell[0];
            else dx0 = 0.0f;
            dx0 = dx0 * dx0;
            for (int dcy = -g->n_neighbors[1]; dcy <= g->n_neighbors[1]; dcy++) {
                int ry = y1 + dcy, iy = 0, y2 = ry;
                if (ry < 0) { iy = -1; y2 = ny + ry; }
                else if (ry >= ny) { iy = 1; y2 = ry - ny; }
                float dx1;
                if (dcy > 0) dx1 = (float)(dcy - 1) * g->L_cell[1];
                else if (dcy < 0) dx1 = (float)(dcy + 1) * g->L_cell[1];
                else dx1 = 0.0f;
                dx1 = dx1 * dx1;
                int first_u[3], last_u[3];
                int tf = cu[c1 * 2] - 2;
                if (tf < 0) { first_u[0] = nuz + tf; last_u[0] = nuz - 1; tf = 0; }
                else { first_u[0] = -1; last_u[0] = -1; }
                first_u[1] = tf;
                int tl = cu[c1 * 2 + 1] + 2;
                if (tl >= nuz) { first_u[2] = 0; last_u[2] = tl - nuz; last_u[1] = nuz - 1; }
                else { first_u[2] = -1; last_u[2] = -1; last_u[1] = tl; }
                int col2  = x2 + y2 * nx;
                int head2 = gr->col_head_cell[col2];
                for (int ii = 0; ii < 3; ii++) {
                    int iz = ii - 1;
                    if (first_u[ii] < 0) continue;
                    int fu = x2 * nuz + y2 * (nuz * nx) + first_u[ii];
                    int lu = x2 * nuz + y2 * (nuz * nx) + last_u[ii];
                    /* reference_faults: the reference's scan (MiniCell.cpp:1062-1076), which
                     * ends at the first empty bin after a filled one and so hides the cells
                     * beyond a z gap of a bin's height; otherwise the engine's window, from the
                     * first to the last filled bin (the same list when no bin inside is empty) */
                    int f = -1, l = -1;
                    for (int u = fu; u <= lu; u++) {
                        if (uni_lo[u] >= 0) {
                            if (f < 0) f = u;
                            l = u;
                        } else if (f >= 0 && reference_faults) {
                            break;
                        }
                    }
                    if (f < 0) continue;
                    fu = f;
                    lu = l;
                    int lo = uni_lo[fu], hi = uni_hi[lu];
                    if (lo > hi || head2 < 0) continue;
                    int first_cell = head2 + lo, last_cell = head2 + hi;
                    /* z indices stay inside column 2, as in the engine */
                    int ncz2 = (gr->col_n_atoms[col2] + OGO_N_ATOM_CELL - 1) / OGO_N_ATOM_CELL;
                    if (last_cell > head2 + ncz2 - 1) last_cell = head2 + ncz2 - 1;
                    for (int c2 = first_cell; c2 <= last_cell; c2++) {
                        float z2t = (float)gr->slot_crd[(c2 * OGO_N_ATOM_CELL + OGO_N_ATOM_CELL - 1) * 3 + 2]
                                    + (float)iz * p->L[2];
                        float z2b = (float)gr->slot_crd[(c2 * OGO_N_ATOM_CELL) * 3 + 2] + (float)iz * p->L[2];
                        float dz;
                        if (z2t < z1b) { dz = z1b - z2t; dz = dz * dz; }
                        else if (z2b > z1t) { dz = z2b - z1t; dz = dz * dz; }
                        else dz = 0.0f;
                        if (dx0 + dx1 + dz > g->cutoff_pair2) continue;
                        if (!valid_pair(c1, c2)) continue;
                        if (n >= cap) {
                            cap *= 2;
                            out->cell1 = (int *)realloc(out->cell1, sizeof(int) * (size_t)cap);
                            out->cell2 = (int *)realloc(out->cell2, sizeof(int) * (size_t)cap);
                            out->image = (int *)realloc(out->image, sizeof(int) * (size_t)cap);
                            out->mask  = (uint64_t *)realloc(out->mask, sizeof(uint64_t) * (size_t)cap);
                        }
                        int img = 0;
                        if (ix == -1) img |= 1; else if (ix == 1) img |= 2;
                        if (iy == -1) img |= 4; else if (iy == 1) img |= 8;
                        if (iz == -1) img |= 16; else if (iz == 1) img |= 32;
                        out->cell1[n] = c1;
                        out->cell2[n] = c2;
                        out->image[n] = img;
                        out->mask[n]  = pair_mask(gr, c1, c2, nb15off, max_nb15off);
                        n++;
                    }
                }
            }
        }
    }
    out->idx_head[n_cells] = n;
    out->n_pairs = n;
    free(uni_lo);
    free(uni_hi);
    free(cu);
    return 0;
}

void ogo_cellpairs_free(ogo_cellpairs *cp) {
    free(cp->idx_head);
    free(cp->cell1);
    free(cp->cell2);
    free(cp->image);
    free(cp->mask);
    memset(cp, 0, sizeof(*cp));
}

/* ------------------------------------------------------- pair energy */

void ogo_zd_constants(double cutoff, float *zcore, float *bcoeff, float *fcoeff) {
    /* ZeroMultipoleSum::set_zms_params with ewald_alpha = 0 (:150-202), real_pw members */
    float c   = (float)cutoff;
    float c2  = c * c;
    float c3  = c2 * c;
    float erc = erfcf(c * 0.0f);
    *fcoeff   = (float)(1.0 / (double)c3);
    *bcoeff   = (float)(0.5 * (double)*fcoeff);
    *zcore    = erc / c + *bcoeff * c2;
}

/* ForceField::calc_pairwise (ForceField.cpp:333-418) + calc_zero02pole_alpha0
 * (ZeroMultipoleSum.cpp:309-332), float arithmetic as compiled by the reference. */
static void calc_pair_f32(float *ev, float *ee, double w[3], const float c1[3], const float c2[3],
                          float p6, float p12, float q1, float q2, double cutoff,
                          float zcore, float bcoeff, float fcoeff) {
    float d[3];
    for (int k = 0; k < 3; k++) d[k] = c1[k] - c2[k];
    float r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    float r  = sqrtf(r2);
    *ev = 0.0f;
    *ee = 0.0f;
    w[0] = w[1] = w[2] = 0.0;
    if ((double)r >= cutoff) return;
    float r_inv   = (float)(1.0 / (double)r);
    float r2_inv  = (float)(1.0 / (double)r2);
    float r3_inv  = r_inv * r2_inv;
    float r6_inv  = r3_inv * r3_inv;
    float r12_inv = r6_inv * r6_inv;
    float t6      = p6 * r6_inv;
    float t12     = p12 * r12_inv;
    *ev           = -t6 + t12;
    float wc      = (float)((double)r2_inv * (-12.0 * (double)t12 + 6.0 * (double)t6));
    float cc      = (float)((double)(q1 * q2) * CHARGE_COEFF);
    *ee           = cc * (r_inv - zcore + bcoeff * r2);
    float gc      = -cc * (r3_inv - fcoeff);
    for (int k = 0; k < 3; k++) {
        float wv = wc * d[k];
        float we = gc * d[k];
        w[k]     = (double)(wv + we);
    }
}

/* PBC::fix_pbc_image, float overload (PBC.cpp:106-121) */
static void fix_image_f(const ogo_pbc *p, float c[3], int image) {
    if (image == 0) return;
    if ((image & 1) == 1) c[0] -= p->L[0];
    else if ((image & 2) == 2) c[0] += p->L[0];
    if ((image & 4) == 4) c[1] -= p->L[1];
    else if ((image & 8) == 8) c[1] += p->L[1];
    if ((image & 16) == 16) c[2] -= p->L[2];
    else if ((image & 32) == 32) c[2] += p->L[2];
}

void ogo_pair_cells_f32(const ogo_pbc *p, const ogo_grid *gr, const ogo_cellpairs *cp,
                        const float *charge, const int *atom_type, int n_types,
                        const float *lj6, const float *lj12, double cutoff,
                        float zcore, float bcoeff, float fcoeff,
                        double *work_slot, double ene[2]) {
    memset(work_slot, 0, sizeof(double) * 3 * (size_t)gr->n_slots);
    ene[0] = ene[1] = 0.0;
    for (int k = 0; k < cp->n_pairs; k++) {
        int c1 = cp->cell1[k], c2 = cp->cell2[k];
        for (int a2 = 0; a2 < OGO_N_ATOM_CELL; a2++) {
            int   g2  = c2 * OGO_N_ATOM_CELL + a2;
            int   id2 = gr->slot_atomid[g2];
            float x2[3] = {(float)gr->slot_crd[g2 * 3], (float)gr->slot_crd[g2 * 3 + 1],
                           (float)gr->slot_crd[g2 * 3 + 2]};
            fix_image_f(p, x2, cp->image[k]);
            for (int a1 = 0; a1 < OGO_N_ATOM_CELL; a1++) {
                if ((cp->mask[k] >> (a2 * OGO_N_ATOM_CELL + a1)) & 1) continue;
                int   g1  = c1 * OGO_N_ATOM_CELL + a1;
                int   id1 = gr->slot_atomid[g1];
                float x1[3] = {(float)gr->slot_crd[g1 * 3], (float)gr->slot_crd[g1 * 3 + 1],
                               (float)gr->slot_crd[g1 * 3 + 2]};
                int   ti = atom_type[id1] * n_types + atom_type[id2];
                float ev, ee;
                double w[3];
                calc_pair_f32(&ev, &ee, w, x1, x2, lj6[ti], lj12[ti], charge[id1], charge[id2], cutoff,
                              zcore, bcoeff, fcoeff);
                ene[0] += (double)ev;
                ene[1] += (double)ee;
                for (int d = 0; d < 3; d++) {
                    work_slot[g1 * 3 + d] += w[d];
                    work_slot[g2 * 3 + d] += -w[d];
                }
            }
        }
    }
}

void ogo_pair_allpairs_f32(const ogo_pbc *p, int n, const double *crd,
                           const float *charge, const int *atom_type, int n_types,
                           const float *lj6, const float *lj12, const int *nb15off, int max_nb15off,
                           double cutoff, float zcore, float bcoeff, float fcoeff,
                           double *work, double ene[2]) {
    memset(work, 0, sizeof(double) * 3 * (size_t)n);
    ene[0] = ene[1] = 0.0;
    for (int a1 = 0; a1 < n; a1++) {
        float x1[3] = {(float)crd[a1 * 3], (float)crd[a1 * 3 + 1], (float)crd[a1 * 3 + 2]};
        for (int a2 = 0; a2 < a1; a2++) {
            float x2[3] = {(float)crd[a2 * 3], (float)crd[a2 * 3 + 1], (float)crd[a2 * 3 + 2]};
            int   excl  = 0;
            for (int k = 0; k < max_nb15off; k++)
                if (nb15off[(size_t)a1 * max_nb15off + k] == a2) excl = 1;
            if (excl) continue;
            int ti = atom_type[a1] * n_types + atom_type[a2];
            for (int d = 0; d < 3; d++) {
                if (x2[d] - x1[d] >= p->L_half[d]) x2[d] -= p->L[d];
                else if (x2[d] - x1[d] <= -p->L_half[d]) x2[d] += p->L[d];
            }
            float  ev, ee;
            double w[3];
            calc_pair_f32(&ev, &ee, w, x1, x2, lj6[ti], lj12[ti], charge[a1], charge[a2], cutoff, zcore,
                          bcoeff, fcoeff);
            ene[0] += (double)ev;
            ene[1] += (double)ee;
            for (int d = 0; d < 3; d++) {
                work[a1 * 3 + d] += w[d];
                work[a2 * 3 + d] -= w[d];
            }
        }
    }
}

/* FP64 LJ + ZD(alpha=0) for one pair: adds gradient on i (=-force) to w, returns 1 if inside. */
static int pair_f64(const double d[3], double p6, double p12, double cc, double rc,
                    double *ev, double *ee, double w[3]) {
    double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    if (r2 >= rc * rc) return 0;
    double r      = sqrt(r2);
    double ri     = 1.0 / r;
    double r2i    = 1.0 / r2;
    double r6i    = r2i * r2i * r2i;
    double t6     = p6 * r6i, t12 = p12 * r6i * r6i;
    double fco    = 1.0 / (rc * rc * rc);
    double bco    = 0.5 * fco;
    double zco    = 1.0 / rc + bco * rc * rc;
    *ev           = t12 - t6;
    *ee           = cc * (ri - zco + bco * r2);
    double wc     = r2i * (-12.0 * t12 + 6.0 * t6) - cc * (ri * r2i - fco);
    for (int k = 0; k < 3; k++) w[k] = wc * d[k];
    return 1;
}

static void add_vir(double vir[9], const double d[3], const double w[3]) {
    /* force on i is -w */
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) vir[a * 3 + b] -= d[a] * w[b];
}

void ogo_pair_allpairs_f64(const double L[3], int n, const double *crd,
                           const double *charge, const int *atom_type, int n_types,
                           const double *lj6, const double *lj12, const int *nb15off, int max_nb15off,
                           double cutoff, double *work, double ene[2], double vir[9]) {
    memset(work, 0, sizeof(double) * 3 * (size_t)n);
    ene[0] = ene[1] = 0.0;
    for (int k = 0; k < 9; k++) vir[k] = 0.0;
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < i; j++) {
            int excl = 0;
            for (int k = 0; k < max_nb15off; k++) {
                int e = nb15off[(size_t)i * max_nb15off + k];
                if (e == -1) break;
                if (e == j) { excl = 1; break; }
            }
            if (excl) continue;
            double d[3];
            for (int k = 0; k < 3; k++) {
                d[k] = crd[i * 3 + k] - crd[j * 3 + k];
                d[k] -= L[k] * nearbyint(d[k] / L[k]);
            }
            int    ti = atom_type[i] * n_types + atom_type[j];
            double ev, ee, w[3];
            if (!pair_f64(d, lj6[ti], lj12[ti], charge[i] * charge[j] * CHARGE_COEFF, cutoff, &ev, &ee, w))
                continue;
            ene[0] += ev;
            ene[1] += ee;
            for (int k = 0; k < 3; k++) {
                work[i * 3 + k] += w[k];
                work[j * 3 + k] -= w[k];
            }
            add_vir(vir, d, w);
        }
    }
}

void ogo_pair_cells_f64(const double L[3], const ogo_grid *gr, const ogo_cellpairs *cp,
                        const double *crd, const double *charge, const int *atom_type, int n_types,
                        const double *lj6, const double *lj12, double cutoff,
                        double *work, double ene[2], double vir[9]) {
    /* work is indexed by original atom id; the caller sizes it [n_atoms*3] */
    ene[0] = ene[1] = 0.0;
    for (int k = 0; k < 9; k++) vir[k] = 0.0;
    for (int k = 0; k < cp->n_pairs; k++) {
        int c1 = cp->cell1[k], c2 = cp->cell2[k];
        for (int a2 = 0; a2 < OGO_N_ATOM_CELL; a2++) {
            int id2 = gr->slot_atomid[c2 * OGO_N_ATOM_CELL + a2];
            for (int a1 = 0; a1 < OGO_N_ATOM_CELL; a1++) {
                if ((cp->mask[k] >> (a2 * OGO_N_ATOM_CELL + a1)) & 1) continue;
                int    id1 = gr->slot_atomid[c1 * OGO_N_ATOM_CELL + a1];
                int    img = cp->image[k];
                double sh[3] = {(img & 1) ? -L[0] : (img & 2) ? L[0] : 0.0,
                                (img & 4) ? -L[1] : (img & 8) ? L[1] : 0.0,
                                (img & 16) ? -L[2] : (img & 32) ? L[2] : 0.0};
                double d[3];
                /* the image recorded with the cell pair, not the minimum image: in small
                 * boxes one column is reached through two images */
                for (int q = 0; q < 3; q++) d[q] = crd[id1 * 3 + q] - (crd[id2 * 3 + q] + sh[q]);
                int    ti = atom_type[id1] * n_types + atom_type[id2];
                double ev, ee, w[3];
                if (!pair_f64(d, lj6[ti], lj12[ti], charge[id1] * charge[id2] * CHARGE_COEFF, cutoff, &ev, &ee,
                              w))
                    continue;
                ene[0] += ev;
                ene[1] += ee;
                for (int q = 0; q < 3; q++) {
                    work[id1 * 3 + q] += w[q];
                    work[id2 * 3 + q] -= w[q];
                }
                add_vir(vir, d, w);
            }
        }
    }
}

double ogo_excess_f32(const ogo_pbc *p, int n_excess, const int *ep, const double *crd,
                      const float *charge, float bcoeff, float fcoeff, double *work) {
    double sum = 0.0;
    for (int k = 0; k < n_excess; k++) {
        int   i = ep[2 * k], j = ep[2 * k + 1];
        float c1[3] = {(float)crd[i * 3], (float)crd[i * 3 + 1], (float)crd[i * 3 + 2]};
        float c2[3] = {(float)crd[j * 3], (float)crd[j * 3 + 1], (float)crd[j * 3 + 2]};
        float d[3];
        diff_minim_f(p, d, c1, c2);
        float r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        float cc = (float)((double)(charge[i] * charge[j]) * CHARGE_COEFF);
        float e  = cc * bcoeff * r2;
        float gc = cc * fcoeff;
        sum += (double)e;
        for (int q = 0; q < 3; q++) {
            double w = (double)(gc * d[q]);
            work[i * 3 + q] += w;
            work[j * 3 + q] -= w;
        }
    }
    return sum;
}

double ogo_excess_f64(const double L[3], int n_excess, const int *ep, const double *crd,
                      const double *charge, double cutoff, double *work, double vir[9]) {
    double sum = 0.0;
    double fco = 1.0 / (cutoff * cutoff * cutoff), bco = 0.5 * fco;
    for (int k = 0; k < n_excess; k++) {
        int    i = ep[2 * k], j = ep[2 * k + 1];
        double d[3], w[3];
        for (int q = 0; q < 3; q++) {
            d[q] = crd[i * 3 + q] - crd[j * 3 + q];
            d[q] -= L[q] * nearbyint(d[q] / L[q]);
        }
        double cc = charge[i] * charge[j] * CHARGE_COEFF;
        double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        sum += cc * bco * r2;
        for (int q = 0; q < 3; q++) {
            w[q] = cc * fco * d[q];
            work[i * 3 + q] += w[q];
            work[j * 3 + q] -= w[q];
        }
        if (vir) add_vir(vir, d, w);
    }
    return sum;
}

double ogo_self_energy(int n, int n_excess, const int *ep, const float *charge, float zcore) {
    double *dw = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    for (int k = 0; k < n_excess; k++) {
        dw[ep[2 * k]] += (double)charge[ep[2 * k + 1]];
        dw[ep[2 * k + 1]] += (double)charge[ep[2 * k]];
    }
    float  mon    = 0.0f;
    double zmcore = (double)zcore;
    float  piew   = 0.0f;
    for (int i = 0; i < n; i++) {
        double q  = (double)charge[i];
        double es = ((double)(-piew * charge[i] * charge[i]) - zmcore * q * (q + dw[i])) * 0.5 * CHARGE_COEFF;
        mon       = (float)((double)mon + es);
    }
    free(dw);
    return (double)mon;
}

int ogo_excess_pairs(int n, const int *nb15off, int max_nb15off, int *out, int cap) {
    int ne = 0;
    for (int i = 0; i < n; i++)
        for (int k = 0; k < max_nb15off; k++) {
            int j = nb15off[(size_t)i * max_nb15off + k];
            if (j == -1) break;
            if (i >= j) continue;
            if (ne >= cap) return -1;
            out[2 * ne] = i;
            out[2 * ne + 1] = j;
            ne++;
        }
    return ne;
}

double ogo_bonds(const ogo_pbc *p, int nb, const int *pairs, const double *k, const double *r0,
                 const double *crd, double *work) {
    double e = 0.0;
    for (int b = 0; b < nb; b++) {
        int    i = pairs[2 * b], j = pairs[2 * b + 1];
        double d[3];
        diff_minim_d(p, d, crd + i * 3, crd + j * 3);
        double r    = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        double dif  = r - r0[b];
        double coef = k[b] * dif;
        e += coef * dif;
        double gc = 2.0 * coef / r;
        for (int q = 0; q < 3; q++) {
            work[i * 3 + q] += d[q] * gc;
            work[j * 3 + q] -= d[q] * gc;
        }
    }
    return e;
}

static void cross3(const double a[3], const double b[3], double c[3]) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

/* ForceField::calc_torsion: the reference's PI constant (CelesteObject.cpp:27) and gmul table
 * (ForceField.cpp:7-17, 2k for even k, 0 otherwise) are part of the arithmetic. */
#define REF_PI 3.14159265
#define REF_EPS 1e-10
double ogo_dihedrals(const ogo_pbc *p, int n, const int *quads, const double *ene, const int *overlaps,
                     const int *symmetry, const double *phase, const double *crd, double *work) {
    double e_sum = 0.0;
    for (int t = 0; t < n; t++) {
        const int a1 = quads[4 * t], a2 = quads[4 * t + 1], a3 = quads[4 * t + 2], a4 = quads[4 * t + 3];
        double w1[3] = {0, 0, 0}, w2[3] = {0, 0, 0}, w3[3] = {0, 0, 0}, e = 0.0;
        if (ene[t] > REF_EPS) {
            double d21[3], d32[3], d43[3], p12[3], p23[3], p123[3];
            diff_minim_d(p, d21, crd + 3 * a2, crd + 3 * a1);
            diff_minim_d(p, d32, crd + 3 * a3, crd + 3 * a2);
            diff_minim_d(p, d43, crd + 3 * a4, crd + 3 * a3);
            cross3(d21, d32, p12);
            cross3(d32, d43, p23);
            double p12_2 = p12[0] * p12[0] + p12[1] * p12[1] + p12[2] * p12[2];
            double p23_2 = p23[0] * p23[0] + p23[1] * p23[1] + p23[2] * p23[2];
            double p12p23 = sqrt(p12_2 * p23_2);
            if (p12p23 > 0.0) {
                double inv = 1.0 / p12p23;
                double s1223 = p12[0] * p23[0] + p12[1] * p23[1] + p12[2] * p23[2];
                double cosp = s1223 * inv;
                if (cosp > 1.0) cosp = 1.0;
                if (cosp < -1.0) cosp = -1.0;
                cross3(p12, p23, p123);
                double phi = acos(cosp);
                if (d32[0] * p123[0] + d32[1] * p123[1] + d32[2] * p123[2] < 0.0) phi = 2.0 * REF_PI - phi;
                const double sym = (double)symmetry[t];
                const double div = 1.0 / (double)overlaps[t];
                e = ene[t] * (1.0 + cos(sym * phi - phase[t])) * div;
                const int nrot = symmetry[t];
                const double gm = (nrot >= 0 && nrot <= 10 && nrot % 2 == 0) ? (double)nrot : 0.0;
                const double sinp = sin(phi);
                const double sf = sin(phase[t]), cf = cos(phase[t]);
                const double sr = sin(sym * phi), cr = cos(sym * phi);
                const double dflim = cf * (sym - gm + gm * cosp);
                const double df0 = cf * sr - sf * cr;
                const double df1 = (REF_EPS <= fabs(sinp)) ? df0 / sinp : dflim;
                const double wc = sym * ene[t] * div * df1 * inv;
                const double r12 = 1.0 / p12_2 * s1223, r23 = 1.0 / p23_2 * s1223;
                double a[3], b[3], c[3], dd[3], f[3], g[3];
                cross3(p23, d32, a);
                cross3(p12, d32, b);
                for (int i = 0; i < 3; i++) w1[i] = wc * (a[i] - r12 * b[i]);
                double d2132[3] = {d21[0] + d32[0], d21[1] + d32[1], d21[2] + d32[2]};
                cross3(d2132, p23, a);
                cross3(d2132, p12, b);
                cross3(p12, d43, c);
                cross3(p23, d43, dd);
                for (int i = 0; i < 3; i++) w2[i] = wc * (a[i] + c[i] - r12 * b[i] - r23 * dd[i]);
                cross3(p12, d32, f);
                cross3(p23, d32, g);
                for (int i = 0; i < 3; i++) w3[i] = wc * (f[i] - r23 * g[i]);
            }
        }
        e_sum += e;
        for (int d = 0; d < 3; d++) {
            work[3 * a1 + d] += w1[d];
            work[3 * a2 + d] += w2[d];
            work[3 * a3 + d] -= w1[d] + w2[d] + w3[d];
            work[3 * a4 + d] += w3[d];
        }
    }
    return e_sum;
}

void ogo_nb14(const ogo_pbc *p, int n, const int *pairs, const int *types, int n_types, const float *lj6,
              const float *lj12, const float *charge, const double *coeff_vdw, const double *coeff_ele,
              const double *crd, double *work, double *e_vdw, double *e_ele) {
    double ev = 0.0, ee = 0.0;
    for (int k = 0; k < n; k++) {
        const int i = pairs[2 * k], j = pairs[2 * k + 1];
        const int tt = types[2 * k] * n_types + types[2 * k + 1];
        double d[3];
        diff_minim_d(p, d, crd + 3 * i, crd + 3 * j);
        const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        const double r2i = 1.0 / r2, ri = sqrt(r2i);
        const double r6i = r2i * r2i * r2i, r12i = r6i * r6i;
        const double t6 = (double)lj6[tt] * r6i, t12 = (double)lj12[tt] * r12i;
        ev += (-t6 + t12) * coeff_vdw[k];
        const double cw = r2i * coeff_vdw[k] * (-12.0 * t12 + 6.0 * t6);
        const double cc = (double)charge[i] * (double)charge[j] * CHARGE_COEFF * coeff_ele[k];
        ee += cc * ri;
        const double ce = -cc * r2i * ri;
        for (int q = 0; q < 3; q++) {
            const double w = cw * d[q] + ce * d[q];
            work[3 * i + q] += w;
            work[3 * j + q] -= w;
        }
    }
    *e_vdw = ev;
    *e_ele = ee;
}

double ogo_angles(const ogo_pbc *p, int na, const int *t, const double *k, const double *t0,
                  const double *crd, double *work) {
    double e = 0.0;
    for (int a = 0; a < na; a++) {
        int    i = t[3 * a], j = t[3 * a + 1], l = t[3 * a + 2];
        double d12[3], d32[3];
        diff_minim_d(p, d12, crd + i * 3, crd + j * 3);
        diff_minim_d(p, d32, crd + l * 3, crd + j * 3);
        double r12_2 = d12[0] * d12[0] + d12[1] * d12[1] + d12[2] * d12[2];
        double r32_2 = d32[0] * d32[0] + d32[1] * d32[1] + d32[2] * d32[2];
        double rr    = sqrt(r12_2 * r32_2);
        double rri   = 1.0 / rr;
        double cost  = (d12[0] * d32[0] + d12[1] * d32[1] + d12[2] * d32[2]) * rri;
        if (cost > 1.0) cost = 1.0;
        if (cost < -1.0) cost = -1.0;
        double th   = acos(cost);
        double dif  = th - t0[a];
        double coef = k[a] * dif;
        e += coef * dif;
        double r12i = 1.0 / r12_2, r32i = 1.0 / r32_2;
        double st   = sin(th);
        if (st < 1e-10) st = 1e-10;
        double gc = -(2.0 * coef) / st;
        for (int q = 0; q < 3; q++) {
            double w1 = gc * (d32[q] * rri - d12[q] * cost * r12i);
            double w2 = gc * (d12[q] * rri - d32[q] * cost * r32i);
            work[i * 3 + q] += w1;
            work[j * 3 + q] -= w1 + w2;
            work[l * 3 + q] += w2;
        }
    }
    return e;
}

/* ---------------------------------------------------------- integrator */

void ogo_update_velocities(ogo_integ *s) {
    memcpy(s->vel, s->vel_next, sizeof(double) * 3 * (size_t)s->n);
    for (int i = 0; i < s->n; i++)
        for (int d = 0; d < 3; d++)
            s->vel_next[i * 3 + d] =
                s->vel[i * 3 + d] + (s->dt * -FORCE_VEL * s->work[i * 3 + d] * (double)s->mass_inv[i]);
}

void ogo_cancel_com(ogo_integ *s, double *v) {
    for (int g = 0; g < s->n_com_groups; g++) {
        double m[3] = {0, 0, 0};
        for (int k = s->com_group_start[g]; k < s->com_group_start[g + 1]; k++) {
            int i = s->com_group_atoms[k];
            for (int d = 0; d < 3; d++) m[d] += v[i * 3 + d] * (double)s->mass[i];
        }
        for (int d = 0; d < 3; d++) m[d] *= (double)s->com_mass_inv[g];
        for (int k = s->com_group_start[g]; k < s->com_group_start[g + 1]; k++) {
            int i = s->com_group_atoms[k];
            for (int d = 0; d < 3; d++) v[i * 3 + d] -= m[d];
        }
    }
}

void ogo_thermostat_scaling(ogo_integ *s) {
    double kp = 0.0;
    for (int i = 0; i < s->n; i++) {
        double vn = 0.0;
        for (int d = 0; d < 3; d++) {
            double vt = s->vel[i * 3 + d] - 0.5 * (s->dt * s->work[i * 3 + d] * FORCE_VEL * (double)s->mass_inv[i]);
            vn += vt * vt;
        }
        kp += (double)s->mass[i] * vn;
    }
    double tcur  = kp * s->temperature_coeff;
    double scale = sqrt(1 + s->dt * s->tau_inv * (s->temperature / tcur - 1));
    for (int i = 0; i < s->n; i++)
        for (int d = 0; d < 3; d++) {
            double vd = s->dt * -FORCE_VEL * s->work[i * 3 + d] * (double)s->mass_inv[i];
            s->vel_next[i * 3 + d] = (2.0 * scale - 1.0) * s->vel[i * 3 + d] + scale * vd;
        }
}

void ogo_update_coordinates(ogo_integ *s) {
    memcpy(s->crd_prev, s->crd, sizeof(double) * 3 * (size_t)s->n);
    for (int i = 0; i < 3 * s->n; i++) s->crd[i] = s->crd_prev[i] + s->vel_next[i] * s->dt;
}

static void shake_pairs(ogo_integ *s, const ogo_pbc *p) {
    for (int c = 0; c < s->n_pair; c++) {
        int    i = s->pair_atoms[2 * c], j = s->pair_atoms[2 * c + 1];
        double d12[3], d12p[3];
        diff_minim_d(p, d12, s->crd + j * 3, s->crd + i * 3);
        diff_minim_d(p, d12p, s->crd_prev + j * 3, s->crd_prev + i * 3);
        double m1 = (double)s->mass_inv[i], m2 = (double)s->mass_inv[j];
        double m12 = m1 + m2;
        double dsq  = d12[0] * d12[0] + d12[1] * d12[1] + d12[2] * d12[2];
        double dsqp = d12p[0] * d12p[0] + d12p[1] * d12p[1] + d12p[2] * d12p[2];
        double dip  = d12[0] * d12p[0] + d12[1] * d12p[1] + d12[2] * d12p[2];
        double va = m12 * m12 * dsqp, vb = m12 * dip, vc = dsq - s->pair_dist2[c];
        double disc = vb * vb - vc * va;
        if (disc < 0.0) disc = 0.0;
        double vg = (vb - sqrt(disc)) / va;
        for (int d = 0; d < 3; d++) {
            s->crd[i * 3 + d] += m1 * vg * d12p[d];
            s->crd[j * 3 + d] -= m2 * vg * d12p[d];
        }
    }
}

static void shake_trios(ogo_integ *s, const ogo_pbc *p) {
    for (int c = 0; c < s->n_trio; c++) {
        int a1 = s->trio_atoms[3 * c], a2 = s->trio_atoms[3 * c + 1], a3 = s->trio_atoms[3 * c + 2];
        double d12[3], d23[3], d31[3], d12p[3], d23p[3], d31p[3];
        double g[6] = {0, 0, 0, 0, 0, 0};
        diff_minim_d(p, d12, s->crd + a1 * 3, s->crd + a2 * 3);
        diff_minim_d(p, d12p, s->crd_prev + a1 * 3, s->crd_prev + a2 * 3);
        diff_minim_d(p, d23, s->crd + a2 * 3, s->crd + a3 * 3);
        diff_minim_d(p, d23p, s->crd_prev + a2 * 3, s->crd_prev + a3 * 3);
        diff_minim_d(p, d31, s->crd + a3 * 3, s->crd + a1 * 3);
        diff_minim_d(p, d31p, s->crd_prev + a3 * 3, s->crd_prev + a1 * 3);
        double m1 = (double)s->mass_inv[a1], m2 = (double)s->mass_inv[a2], m3 = (double)s->mass_inv[a3];
        double c11 = m1 + m2, c12 = -m2, c13 = -m1;
        double c21 = -m2, c22 = m2 + m3, c23 = -m3;
        double c31 = -m1, c32 = -m3, c33 = m3 + m1;
        const double *td = s->trio_dist2 + 3 * c;
        for (int it = 0; it < s->shake_max_loops; it++) {
            for (int d = 0; d < 3; d++) {
                d12[d] += (c11 * d12p[d] * g[0] + c12 * d23p[d] * g[1] + c13 * d31p[d] * g[2]);
                d23[d] += (c21 * d12p[d] * g[0] + c22 * d23p[d] * g[1] + c23 * d31p[d] * g[2]);
                d31[d] += (c31 * d12p[d] * g[0] + c32 * d23p[d] * g[1] + c33 * d31p[d] * g[2]);
            }
#define DOT(a, b) (a[0] * b[0] + a[1] * b[1] + a[2] * b[2])
            double f11 = 2.0 * c11 * DOT(d12, d12p), f12 = 2.0 * c12 * DOT(d12, d23p), f13 = 2.0 * c13 * DOT(d12, d31p);
            double f21 = 2.0 * c21 * DOT(d23, d12p), f22 = 2.0 * c22 * DOT(d23, d23p), f23 = 2.0 * c23 * DOT(d23, d31p);
            double f31 = 2.0 * c31 * DOT(d31, d12p), f32 = 2.0 * c32 * DOT(d31, d23p), f33 = 2.0 * c33 * DOT(d31, d31p);
            double df[3] = {td[0] - DOT(d12, d12), td[1] - DOT(d23, d23), td[2] - DOT(d31, d31)};
#undef DOT
            if (fabs(df[0] / td[0]) < s->shake_tol && fabs(df[1] / td[1]) < s->shake_tol &&
                fabs(df[2] / td[2]) < s->shake_tol)
                break;
            double det = 1.0 / (f11 * f22 * f33 + f12 * f23 * f31 + f13 * f21 * f32 - f11 * f23 * f32 -
                                f12 * f21 * f33 - f13 * f22 * f31);
            double b11 = f22 * f33 - f23 * f32, b12 = f32 * f13 - f33 * f12, b13 = f12 * f23 - f13 * f22;
            double b21 = f23 * f31 - f21 * f33, b22 = f33 * f11 - f31 * f13, b23 = f13 * f21 - f11 * f23;
            double b31 = f21 * f32 - f22 * f31, b32 = f31 * f12 - f32 * f11, b33 = f11 * f22 - f12 * f21;
            g[0] = (b11 * df[0] + b12 * df[1] + b13 * df[2]) * det;
            g[1] = (b21 * df[0] + b22 * df[1] + b23 * df[2]) * det;
            g[2] = (b31 * df[0] + b32 * df[1] + b33 * df[2]) * det;
            g[3] += g[0];
            g[4] += g[1];
            g[5] += g[2];
        }
        for (int d = 0; d < 3; d++) {
            s->crd[a1 * 3 + d] += m1 * (g[3] * d12p[d] - g[5] * d31p[d]);
            s->crd[a2 * 3 + d] += m2 * (-g[3] * d12p[d] + g[4] * d23p[d]);
            s->crd[a3 * 3 + d] += m3 * (-g[4] * d23p[d] + g[5] * d31p[d]);
        }
    }
}

/* ConstraintObject::calc_linear_eq (Constraint.cpp:141-202): elimination with the pivot
 * permutation applied to the column index, a[6][6] overwritten.  Returns 1 if singular. */
static int solve6(double a[6][6], double x[6], const double b[6]) {
    int piv[6] = {0, 1, 2, 3, 4, 5};
    for (int i = 0; i < 6; i++) {
        int idx = i;
        double mx = fabs(a[i][piv[i]]);
        for (int j = i + 1; j < 6; j++) {
            double t = fabs(a[i][piv[j]]);
            if (t > mx) { idx = j; mx = t; }
        }
        if (idx != i) { int t = piv[i]; piv[i] = piv[idx]; piv[idx] = t; }
        if (fabs(a[i][piv[i]]) < 1e-30) return 1;
        a[i][piv[i]] = 1.0 / a[i][piv[i]];
        for (int j = i + 1; j < 6; j++) {
            a[i][piv[j]] *= a[i][piv[i]];
            for (int k = i + 1; k < 6; k++) a[k][piv[j]] -= a[i][piv[j]] * a[k][piv[i]];
        }
    }
    for (int i = 0; i < 6; i++) {
        double v = b[piv[i]];
        for (int j = 0; j < i; j++) v -= a[j][piv[i]] * x[j];
        x[i] = v;
    }
    for (int i = 5; i >= 0; i--) {
        double v = x[i];
        for (int j = i + 1; j < 6; j++) v -= a[j][piv[i]] * x[j];
        x[i] = v * a[i][piv[i]];
    }
    return 0;
}

/* ConstraintShake::shake_quad (ConstraintShake.cpp:151-276): one centre and three partners,
 * six distances (Constraint.cpp:4 pair order), Newton steps with a 6x6 solve. */
static void shake_quads(ogo_integ *s, const ogo_pbc *p) {
    static const int PI2[6][2] = {{0, 1}, {1, 2}, {2, 0}, {3, 0}, {2, 3}, {1, 3}};
    for (int c = 0; c < s->n_quad; c++) {
        const int *at = s->quad_atoms + 4 * c;
        const double *qd = s->quad_dist2 + 6 * c;
        double mi[4];
        for (int i = 0; i < 4; i++) mi[i] = (double)s->mass_inv[at[i]];
        const double w[6][6] = {{mi[0] + mi[1], -mi[1], -mi[0], -mi[0], 0.0, -mi[1]},
                                {-mi[1], mi[1] + mi[2], -mi[2], 0.0, -mi[2], mi[1]},
                                {-mi[0], -mi[2], mi[2] + mi[0], mi[0], mi[2], 0.0},
                                {-mi[0], 0.0, mi[0], mi[3] + mi[0], -mi[3], -mi[3]},
                                {0.0, -mi[2], mi[2], -mi[3], mi[2] + mi[3], mi[3]},
                                {-mi[1], mi[1], 0.0, -mi[3], mi[3], mi[1] + mi[3]}};
        double dc[6][3], dp[6][3];
        for (int k = 0; k < 6; k++) {
            diff_minim_d(p, dc[k], s->crd + 3 * at[PI2[k][0]], s->crd + 3 * at[PI2[k][1]]);
            diff_minim_d(p, dp[k], s->crd_prev + 3 * at[PI2[k][0]], s->crd_prev + 3 * at[PI2[k][1]]);
        }
        double coef[6] = {0, 0, 0, 0, 0, 0}, coef_post[6] = {0, 0, 0, 0, 0, 0};
        for (int it = 0; it < s->shake_max_loops; it++) {
            for (int k = 0; k < 6; k++) coef[k] = coef_post[k];
            double dv[6][3];
            for (int i = 0; i < 6; i++) {
                for (int d = 0; d < 3; d++) dv[i][d] = dc[i][d];
                for (int j = 0; j < 6; j++)
                    for (int d = 0; d < 3; d++) dv[i][d] += w[j][i] * dp[j][d] * coef[j];
            }
            double g[6][6];
            for (int i = 0; i < 6; i++)
                for (int j = 0; j < 6; j++)
                    g[i][j] = 2.0 * w[j][i] * (dv[j][0] * dp[i][0] + dv[j][1] * dp[i][1] + dv[j][2] * dp[i][2]);
            int conv = 1;
            double sd[6];
            for (int i = 0; i < 6; i++) {
                double nrm = dv[i][0] * dv[i][0] + dv[i][1] * dv[i][1] + dv[i][2] * dv[i][2];
                sd[i] = qd[i] - nrm;
                conv = conv && (fabs(sd[i] / qd[i]) < s->shake_tol);
            }
            if (conv) break;
            double rhs[6];
            for (int i = 0; i < 6; i++) {
                rhs[i] = sd[i];
                for (int j = 0; j < 6; j++) rhs[i] += g[j][i] * coef[j];
            }
            solve6(g, coef_post, rhs);
        }
        for (int d = 0; d < 3; d++) {
            s->crd[3 * at[0] + d] += mi[0] * (coef[0] * dp[0][d] - coef[2] * dp[2][d] - coef[3] * dp[3][d]);
            s->crd[3 * at[1] + d] += mi[1] * (-coef[0] * dp[0][d] + coef[1] * dp[1][d] + coef[5] * dp[5][d]);
            s->crd[3 * at[2] + d] += mi[2] * (-coef[1] * dp[1][d] + coef[2] * dp[2][d] + coef[4] * dp[4][d]);
            s->crd[3 * at[3] + d] += mi[3] * (coef[3] * dp[3][d] - coef[4] * dp[4][d] - coef[5] * dp[5][d]);
        }
    }
}

void ogo_shake(ogo_integ *s, const ogo_pbc *p) {
    shake_pairs(s, p);
    shake_trios(s, p);
    shake_quads(s, p);
}

void ogo_set_velocity_from_crd(ogo_integ *s) {
    double dti = 1.0 / s->dt;
    for (int i = 0; i < 3 * s->n; i++) s->vel_next[i] = (s->crd[i] - s->crd_prev[i]) * dti;
}

int ogo_thermostat_with_shake(ogo_integ *s, const ogo_pbc *p) {
    const int n3 = 3 * s->n;
    double dt = s->dt, dtisq = 1.0 / (dt * dt);
    int converge = 0;
    memcpy(s->buf_crd, s->crd, sizeof(double) * (size_t)n3);
    for (int it = 0; it < s->thermo_max_loops; it++) {
        ogo_shake(s, p);
        double kp = 0.0;
        for (int i = 0; i < s->n; i++) {
            double vn = 0.0;
            for (int d = 0; d < 3; d++) {
                double vt = (s->vel_next[i * 3 + d] + s->vel[i * 3 + d]) * 0.5;
                vn += vt * vt;
            }
            kp += vn * (double)s->mass[i];
        }
        double tcur = kp * s->temperature_coeff;
        if (it == s->thermo_max_loops - 1) break;
        if (fabs(tcur - s->temperature) / s->temperature < s->thermo_tol) { converge = 1; break; }
        kp = 0.0;
        for (int i = 0; i < s->n; i++) {
            double vn = 0.0;
            for (int d = 0; d < 3; d++) {
                int    k  = i * 3 + d;
                double vd = -FORCE_VEL * s->work[k] * (double)s->mass_inv[i] + (s->crd[k] - s->buf_crd[k]) * dtisq;
                s->vel_next[k] = s->vel[k] + 0.5 * dt * vd;
                double vt      = s->vel_next[k];
                vn += vt * vt;
            }
            kp += (double)s->mass[i] * vn;
        }
        tcur = kp * s->temperature_coeff;
        double scale = sqrt(s->temperature / tcur);
        for (int i = 0; i < s->n; i++)
            for (int d = 0; d < 3; d++) {
                int    k  = i * 3 + d;
                double vd = -FORCE_VEL * s->work[k] * (double)s->mass_inv[i] + (s->crd[k] - s->buf_crd[k]) * dtisq;
                s->vel_next[k] = (2.0 * scale - 1.0) * s->vel[k] + scale * dt * vd;
            }
        ogo_cancel_com(s, s->vel_next);
        for (int k = 0; k < n3; k++) s->crd[k] = s->crd_prev[k] + dt * s->vel_next[k];
    }
    return converge;
}

void ogo_revise_pbc(const ogo_pbc *p, int n, double *crd) {
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) {
            if (crd[i * 3 + d] >= (double)p->upper[d]) crd[i * 3 + d] -= (double)p->L[d];
            else if (crd[i * 3 + d] < (double)p->lower[d]) crd[i * 3 + d] += (double)p->L[d];
        }
}

void ogo_move_grid(const ogo_grid *gr, int n, const double *crd, const double *crd_prev, double *slot_crd) {
    for (int i = 0; i < n; i++) {
        int s = gr->atomids_rev[i];
        for (int d = 0; d < 3; d++) slot_crd[s * 3 + d] += crd[i * 3 + d] - crd_prev[i * 3 + d];
    }
}

double ogo_kinetic(const ogo_integ *s, double *vj) {
    double kp = 0.0;
    for (int i = 0; i < s->n; i++) {
        double ka = 0.0;
        for (int d = 0; d < 3; d++) {
            double v = (s->vel[i * 3 + d] + s->vel_next[i * 3 + d]) * 0.5;
            if (vj) vj[i * 3 + d] = v;
            ka += v * v;
        }
        kp += ka * (double)s->mass[i];
    }
    return kp * KINETIC_COEFF;
}

double ogo_mcmd_scale(double lambda, double lo, double hi, int order, const double *coef, double temperature,
                      int n, double *work) {
    double param = lambda;
    if (lambda <= lo) param = lo;
    else if (lambda >= hi) param = hi;
    double dlnp = coef[0], t = 1.0;
    for (int i = 1; i < order + 1; i++) {
        t *= param;
        dlnp += coef[i] * t;
    }
    double k   = (GAS_CONST / JOULE_CAL) * 1e-3 * temperature;
    double dew = k * dlnp;
    for (int i = 0; i < 3 * n; i++) work[i] *= dew;
    return dew;
}

/* ------------------------------------------------------------------ V-McMD transitions */

/* std::mt19937::seed (the C++ standard's [rand.eng.mers] initialisation): x0 = value,
 * x_i = 1812433253 * (x_{i-1} xor (x_{i-1} >> 30)) + i; the next draw twists first. */
void ogo_mt_seed(uint32_t *st, uint32_t seed) {
    st[0] = seed;
    for (uint32_t i = 1; i < 624; i++) st[i] = 1812433253u * (st[i - 1] ^ (st[i - 1] >> 30)) + i;
    st[624] = 624;
}

/* One draw of mt19937 (Matsumoto & Nishimura 1998, genrand_int32), written word by word. */
uint32_t ogo_mt_next(uint32_t *st) {
    if (st[624] >= 624) {
        for (int k = 0; k < 624; k++) {
            uint32_t y = (st[k] & 0x80000000u) | (st[(k + 1) % 624] & 0x7fffffffu);
            st[k] = st[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        st[624] = 0;
    }
    uint32_t y = st[st[624]++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

static int vs_in_range(const double *lam, int v, double lambda) { /* Extend.cpp:53-55 */
    return lambda >= lam[2 * v] && lambda <= lam[2 * v + 1];
}

/* ExtendedVMcMD::trial_transition (Extend.cpp:160-177); Random::operator() = draw / max. */
static int vs_trial(int n_vs, const double *lam, const double *prob, int src, int rel, double lambda,
                    uint32_t *st) {
    if (!vs_in_range(lam, src, lambda)) return src;
    if (src == 0 && rel == -1) return src;
    if (src == n_vs - 1 && rel == 1) return src;
    int up_down = rel == -1 ? 0 : rel;
    if (vs_in_range(lam, src + rel, lambda)) {
        double r = ogo_mt_next(st) / (double)0xffffffffu;
        if (r > (1.0 - prob[2 * src + up_down])) return src + rel;
    }
    return src;
}

int ogo_vmcmd_transition(int n_vs, const double *lam, const double *prob, int cur, double lambda, uint32_t *st) {
    int dest = vs_trial(n_vs, lam, prob, cur, 1, lambda, st);   /* Extend.cpp:144-158 */
    if (dest != cur) return dest;
    return vs_trial(n_vs, lam, prob, cur, -1, lambda, st);
}

/* ------------------------------------------------ other electrostatics / nonbond models */

#define OGO_PI 3.14159265                /* CelesteObject.cpp:27 */
#define OGO_EPS 1e-10                    /* CelesteObject.cpp:30 */
#define OGO_ELEM_CHARGE 1.60217657e-19   /* CelesteObject.cpp:32 */
#define OGO_AVOGADRO 6.0221413e23        /* CelesteObject.cpp:33 */
#define OGO_PERMITTIVITY 8.85418782e-12  /* CelesteObject.cpp:34 */
#define OGO_BOLTZMAN 1.380658e-23        /* CelesteObject.cpp:39 */

/* ZeroMultipoleSum::set_zms_params (ZeroMultipoleSum.cpp:108-202): members are float, the
 * literals double, so each expression is evaluated as the C++ code evaluates it. */
void ogo_ele_init(ogo_ele *m, int mode, double alpha, double cutoff, double dh_dielectric,
                  double dh_ionic_strength, double dh_temperature) {
    memset(m, 0, sizeof(*m));
    m->mode = mode;
    m->alpha = (float)alpha;
    m->cutoff = (float)cutoff;
    const float c = m->cutoff, a = m->alpha;
    const float c2 = c * c, c3 = c2 * c, c4 = c2 * c2, c5 = c3 * c2, c6 = c3 * c3, c7 = c3 * c4;
    const float tmp = c * a;
    const float erc = erfcf(tmp);
    const float expterm = expf(-tmp * tmp);
    float fcoeff, bcoeff, hzqrc, d1, d2, d3, d4, piewald = 0.0f;
    m->alpha0 = (double)a < OGO_EPS;
    if (m->alpha0) {
        fcoeff = (float)(1.0 / c3);
        bcoeff = (float)(0.5 * fcoeff);
        hzqrc = (float)(2.0 / c3);
        d1 = (float)(1.0 / c2);
        d2 = (float)(2.0 / c3);
        d3 = (float)(6.0 / c4);
        d4 = (float)(24.0 / c5);
    } else {
        const float root_pi = (float)sqrt(OGO_PI);
        piewald = (float)(2.0 / root_pi * a);
        fcoeff = erc / c3 + piewald * expterm / c2;
        bcoeff = (float)(0.5 * fcoeff);
        const float t3 = tmp * tmp * tmp, t5 = t3 * tmp * tmp, t7 = t5 * tmp * tmp;
        hzqrc = (float)((erc + expterm * (tmp + t3) * 2.0 / root_pi) * 2.0 / c3);
        d1 = (float)((erc + expterm * tmp * 2.0 / root_pi) / c2);
        d2 = (float)((erc + expterm * (tmp + t3) * 2.0 / root_pi) * 2.0 / c3);
        d3 = (float)((erc + expterm * (tmp + 2.0 / 3.0 * t3 + 2.0 / 3.0 * t5) * 2.0 / root_pi) * 6.0 / c4);
        /* "+ 1.0 / 3.0 + tmp_7" as the reference writes it */
        d4 = (float)((erc + expterm * (tmp + 2.0 / 3.0 * t3 + 1.0 / 6.0 * t5 + 1.0 / 3.0 + t7) * 2.0 / root_pi) * 24.0 /
                     c5);
    }
    m->fcoeff = fcoeff;
    m->bcoeff = bcoeff;
    m->piewald = piewald;
    m->zqcoeff2 = (float)(-3.0 / 4.0 * fcoeff - hzqrc / 4.0);
    m->zqcoeff4 = (float)(fcoeff / 8.0 / c2 + hzqrc / 8.0 / c2);
    m->zqcoeff22 = (float)(2.0 * m->zqcoeff2);
    m->zqcoeff44 = (float)(4.0 * m->zqcoeff4);
    m->zocoeff2 = (float)(-15.0 / 16.0 * d1 / c - 7.0 / 16.0 * d2 - 1.0 / 16.0 * d3 * c);
    m->zocoeff4 = (float)(5.0 / 16.0 * d1 / c3 + 5.0 / 16.0 * d2 / c2 + 1.0 / 16.0 * d3 / c);
    m->zocoeff6 = (float)(-1.0 / 16.0 * d1 / c5 - 1.0 / 16.0 * d2 / c4 - 1.0 / 48.0 * d3 / c3);
    m->zocoeff22 = (float)(2.0 * m->zocoeff2);
    m->zocoeff44 = (float)(4.0 * m->zocoeff4);
    m->zocoeff66 = (float)(6.0 * m->zocoeff6);
    m->zhcoeff2 = (float)(-35.0 / 32.0 * d1 / c - 19.0 / 32.0 * d2 - 1.0 / 96.0 * d4 * c2 - 1.0 / 8.0 * d3 * c);
    m->zhcoeff4 = (float)(1.0 / 64.0 * d4 + 35.0 / 64.0 * d1 / c3 + 35.0 / 64.0 * d2 / c2 + 5.0 / 32.0 * d3 / c);
    m->zhcoeff6 = (float)(-7.0 / 32.0 * d1 / c5 - 7.0 / 32.0 * d2 / c4 - 1.0 / 12.0 * d3 / c3 - 1.0 / 96.0 * d4 / c2);
    m->zhcoeff8 = (float)(5.0 / 128.0 * d2 / c6 + 5.0 / 128.0 * d1 / c7 + 1.0 / 64.0 * d3 / c5 + 1.0 / 384.0 * d4 / c4);
    m->zhcoeff22 = (float)(2.0 * m->zhcoeff2);
    m->zhcoeff44 = (float)(4.0 * m->zhcoeff4);
    m->zhcoeff66 = (float)(6.0 * m->zhcoeff6);
    m->zhcoeff88 = (float)(8.0 * m->zhcoeff8);
    m->zcore = erc / c + bcoeff * c2;
    m->zqcore = erc / c - m->zqcoeff2 * c2 - m->zqcoeff4 * c4;
    m->zocore = erc / c - m->zocoeff2 * c2 - m->zocoeff4 * c4 - m->zocoeff6 * c6;
    m->zhcore = erc / c - m->zhcoeff2 * c2 - m->zhcoeff4 * c4 - m->zhcoeff6 * c6 - m->zhcoeff8 * c6 * c2;
    switch (mode) {  /* ZeroMultipoleSum::cal_self_energy (ZeroMultipoleSum.cpp:71-77) */
        case OGO_ELE_ZD: m->zmcore = m->zcore; break;
        case OGO_ELE_ZQ: m->zmcore = m->zqcore; break;
        case OGO_ELE_ZO: m->zmcore = m->zocore; break;
        case OGO_ELE_ZH: m->zmcore = m->zhcore; break;
        default: m->zmcore = 0.0f;
    }
    if (mode == OGO_ELE_DH) { /* the constructor's members (ZeroMultipoleSum.cpp:20-24) */
        m->dielectric_inv = (float)(1.0 / dh_dielectric);
        m->debye_length_inv =
            (float)(1.0 / (sqrt(OGO_PERMITTIVITY * dh_dielectric * OGO_BOLTZMAN * dh_temperature /
                                (2 * OGO_AVOGADRO * OGO_ELEM_CHARGE * OGO_ELEM_CHARGE * dh_ionic_strength)) *
                           1e10));
    }
}

void ogo_ele_init64(ogo_ele64 *m, int mode, double alpha, double cutoff, double dh_dielectric,
                    double dh_ionic_strength, double dh_temperature) {
    memset(m, 0, sizeof(*m));
    m->mode = mode;
    m->alpha = alpha;
    m->cutoff = cutoff;
    const double c = cutoff, a = alpha;
    const double c2 = c * c, c3 = c2 * c, c4 = c2 * c2, c5 = c3 * c2, c6 = c3 * c3, c7 = c3 * c4;
    const double tmp = c * a, erc = erfc(tmp), expterm = exp(-tmp * tmp);
    double hzqrc, d1, d2, d3, d4;
    m->alpha0 = a < OGO_EPS;
    if (m->alpha0) {
        m->fcoeff = 1.0 / c3;
        hzqrc = 2.0 / c3;
        d1 = 1.0 / c2;
        d2 = 2.0 / c3;
        d3 = 6.0 / c4;
        d4 = 24.0 / c5;
    } else {
        const double root_pi = sqrt(OGO_PI);
        m->piewald = 2.0 / root_pi * a;
        m->fcoeff = erc / c3 + m->piewald * expterm / c2;
        const double t3 = tmp * tmp * tmp, t5 = t3 * tmp * tmp, t7 = t5 * tmp * tmp;
        hzqrc = (erc + expterm * (tmp + t3) * 2.0 / root_pi) * 2.0 / c3;
        d1 = (erc + expterm * tmp * 2.0 / root_pi) / c2;
        d2 = (erc + expterm * (tmp + t3) * 2.0 / root_pi) * 2.0 / c3;
        d3 = (erc + expterm * (tmp + 2.0 / 3.0 * t3 + 2.0 / 3.0 * t5) * 2.0 / root_pi) * 6.0 / c4;
        d4 = (erc + expterm * (tmp + 2.0 / 3.0 * t3 + 1.0 / 6.0 * t5 + 1.0 / 3.0 + t7) * 2.0 / root_pi) * 24.0 / c5;
    }
    const double f = m->fcoeff;
    m->bcoeff = 0.5 * f;
    m->zqcoeff2 = -3.0 / 4.0 * f - hzqrc / 4.0;
    m->zqcoeff4 = f / 8.0 / c2 + hzqrc / 8.0 / c2;
    m->zqcoeff22 = 2.0 * m->zqcoeff2;
    m->zqcoeff44 = 4.0 * m->zqcoeff4;
    m->zocoeff2 = -15.0 / 16.0 * d1 / c - 7.0 / 16.0 * d2 - 1.0 / 16.0 * d3 * c;
    m->zocoeff4 = 5.0 / 16.0 * d1 / c3 + 5.0 / 16.0 * d2 / c2 + 1.0 / 16.0 * d3 / c;
    m->zocoeff6 = -1.0 / 16.0 * d1 / c5 - 1.0 / 16.0 * d2 / c4 - 1.0 / 48.0 * d3 / c3;
    m->zocoeff22 = 2.0 * m->zocoeff2;
    m->zocoeff44 = 4.0 * m->zocoeff4;
    m->zocoeff66 = 6.0 * m->zocoeff6;
    m->zhcoeff2 = -35.0 / 32.0 * d1 / c - 19.0 / 32.0 * d2 - 1.0 / 96.0 * d4 * c2 - 1.0 / 8.0 * d3 * c;
    m->zhcoeff4 = 1.0 / 64.0 * d4 + 35.0 / 64.0 * d1 / c3 + 35.0 / 64.0 * d2 / c2 + 5.0 / 32.0 * d3 / c;
    m->zhcoeff6 = -7.0 / 32.0 * d1 / c5 - 7.0 / 32.0 * d2 / c4 - 1.0 / 12.0 * d3 / c3 - 1.0 / 96.0 * d4 / c2;
    m->zhcoeff8 = 5.0 / 128.0 * d2 / c6 + 5.0 / 128.0 * d1 / c7 + 1.0 / 64.0 * d3 / c5 + 1.0 / 384.0 * d4 / c4;
    m->zhcoeff22 = 2.0 * m->zhcoeff2;
    m->zhcoeff44 = 4.0 * m->zhcoeff4;
    m->zhcoeff66 = 6.0 * m->zhcoeff6;
    m->zhcoeff88 = 8.0 * m->zhcoeff8;
    m->zcore = erc / c + m->bcoeff * c2;
    m->zqcore = erc / c - m->zqcoeff2 * c2 - m->zqcoeff4 * c4;
    m->zocore = erc / c - m->zocoeff2 * c2 - m->zocoeff4 * c4 - m->zocoeff6 * c6;
    m->zhcore = erc / c - m->zhcoeff2 * c2 - m->zhcoeff4 * c4 - m->zhcoeff6 * c6 - m->zhcoeff8 * c6 * c2;
    m->zmcore = mode == OGO_ELE_ZD ? m->zcore : mode == OGO_ELE_ZQ ? m->zqcore : mode == OGO_ELE_ZO ? m->zocore
              : mode == OGO_ELE_ZH ? m->zhcore : 0.0;
    if (mode == OGO_ELE_DH) {
        m->dielectric_inv = 1.0 / dh_dielectric;
        m->debye_length_inv = 1.0 / (sqrt(OGO_PERMITTIVITY * dh_dielectric * OGO_BOLTZMAN * dh_temperature /
                                          (2 * OGO_AVOGADRO * OGO_ELEM_CHARGE * OGO_ELEM_CHARGE * dh_ionic_strength)) *
                                     1e10);
    }
}

/* The pair functions of ZeroMultipoleSum.cpp:309-455 (func_calc_zms), float. */
static void ele_pair_f(const ogo_ele *m, float *e, float *g, float r, float r2, float ri, float r2i, float r3i,
                       float cc) {
    const float r4 = r2 * r2, r6 = r4 * r2, r8 = r4 * r4;
    if (m->mode == OGO_ELE_DH) {
        const float ld = expf(-r * m->debye_length_inv);
        *e = cc * ri * m->dielectric_inv * ld;
        *g = -*e * (ri + m->debye_length_inv);
        return;
    }
    float erc = 1.0f, ex = 0.0f;
    if (!m->alpha0) {
        const float t = r * m->alpha;
        erc = erfcf(t);
        ex = m->piewald * expf(-t * t) * r2i;
    }
    switch (m->mode) {
        case OGO_ELE_ZD:
            if (m->alpha0) {
                *e = cc * (ri - m->zcore + m->bcoeff * r2);
                *g = -cc * (r3i - m->fcoeff);
            } else {
                *e = cc * (ri * erc - m->zcore + m->bcoeff * r2);
                *g = -cc * (erc * r3i + ex - m->fcoeff);
            }
            break;
        case OGO_ELE_ZQ:
            if (m->alpha0) {
                *e = cc * (ri - m->zqcore - m->zqcoeff2 * r2 - m->zqcoeff4 * r4);
                *g = -cc * (r3i + m->zqcoeff22 + m->zqcoeff44 * r2);
            } else {
                *e = cc * (ri * erc - m->zqcore - m->zqcoeff2 * r2 - m->zqcoeff4 * r4);
                *g = -cc * (r3i * erc + ex + m->zqcoeff22 + m->zqcoeff44 * r2);
            }
            break;
        case OGO_ELE_ZO:
            if (m->alpha0) {
                *e = cc * (ri - m->zocore - m->zocoeff2 * r2 - m->zocoeff4 * r4 - m->zocoeff6 * r6);
                *g = -cc * (r3i + m->zocoeff22 + m->zocoeff44 * r2 + m->zocoeff66 * r4);
            } else {  /* gradient with the hexadecapole coefficients (ZeroMultipoleSum.cpp:396-398) */
                *e = cc * (ri * erc - m->zocore - m->zocoeff2 * r2 - m->zocoeff4 * r4 - m->zocoeff6 * r6);
                *g = -cc * (r3i * erc + ex + m->zhcoeff22 + m->zhcoeff44 * r2 + m->zhcoeff66 * r4);
            }
            break;
        default:  /* OGO_ELE_ZH */
            if (m->alpha0) {
                *e = cc * (ri - m->zhcore - m->zhcoeff2 * r2 - m->zhcoeff4 * r4 - m->zhcoeff6 * r6 - m->zhcoeff8 * r8);
                *g = -cc * (r3i + m->zhcoeff22 + m->zhcoeff44 * r2 + m->zhcoeff66 * r4 + m->zhcoeff88 * r6);
            } else {
                *e = cc * (ri * erc - m->zhcore - m->zhcoeff2 * r2 - m->zhcoeff4 * r4 - m->zhcoeff6 * r6 -
                           m->zhcoeff8 * r8);
                *g = -cc * (r3i * erc + ex + m->zhcoeff22 + m->zhcoeff44 * r2 + m->zhcoeff66 * r4 + m->zhcoeff88 * r6);
            }
    }
}

/* The excess functions (func_calc_zms_excess, ZeroMultipoleSum.cpp:204-307; calc_null for
 * Debye-Hueckel), float; r4 of the octupole alpha = 0 form is a double in the reference. */
static void ele_excess_f(const ogo_ele *m, float *e, float *g, float r, float r2, float ri, float r2i, float r3i,
                         float cc) {
    if (m->mode == OGO_ELE_DH) {
        *e = 0.0f;
        *g = 0.0f;
        return;
    }
    float erc = 1.0f, erfn = 0.0f, ex = 0.0f;
    if (!m->alpha0) {
        const float t = m->alpha * r;
        erc = erfcf(t);
        erfn = (float)(1.0 - erc);
        ex = m->piewald * expf(-t * t) * r2i;
    }
    const float r4 = r2 * r2;
    switch (m->mode) {
        case OGO_ELE_ZD:
            if (m->alpha0) {
                *e = cc * m->bcoeff * r2;
                *g = cc * m->fcoeff;
            } else {  /* "-errorfn * r12" as written (ZeroMultipoleSum.cpp:215) */
                *e = cc * (-erfn * r + m->bcoeff * r2);
                *g = -cc * (erc * r3i + ex - m->fcoeff - r3i);
            }
            break;
        case OGO_ELE_ZQ:
            if (m->alpha0) {
                *e = cc * (-m->zqcoeff2 * r2 - m->zqcoeff4 * r2 * r2);
                *g = -cc * (m->zqcoeff22 + m->zqcoeff44 * r2);
            } else {
                *e = cc * (-erfn * ri - m->zqcoeff2 * r2 - m->zqcoeff4 * r2 * r2);
                *g = -cc * (erc * r3i + ex + m->zqcoeff22 + m->zqcoeff44 * r2 - r3i);
            }
            break;
        case OGO_ELE_ZO:
            if (m->alpha0) {
                const double r4d = (double)(r2 * r2);  /* a float product stored in a double */
                *e = (float)(cc * (-m->zocoeff2 * r2 - m->zocoeff4 * r4d - m->zocoeff6 * r4d * r));
                *g = (float)(-cc * (m->zocoeff22 + m->zocoeff44 * r2 + m->zocoeff66 * r4d));
            } else {
                *e = cc * (-erfn * ri - m->zocoeff2 * r2 - m->zocoeff4 * r4 - m->zocoeff6 * r4 * r);
                *g = -cc * (erc * r3i + ex + m->zocoeff22 + m->zocoeff44 * r2 + m->zocoeff66 * r4 - r3i);
            }
            break;
        default: {  /* OGO_ELE_ZH */
            const float r6 = r4 * r2, r8 = r4 * r4;
            if (m->alpha0) {
                *e = cc * (-m->zhcoeff2 * r2 - m->zhcoeff4 * r4 - m->zhcoeff6 * r6 - m->zhcoeff8 * r8);
                *g = -cc * (m->zhcoeff22 + m->zhcoeff44 * r2 + m->zhcoeff66 * r2 + m->zhcoeff88 * r6 - r3i);
            } else {
                *e = cc * (-erfn * ri - m->zhcoeff2 * r2 - m->zhcoeff4 * r4);
                *g = -cc * (erc * r3i + ex + m->zhcoeff22 + m->zhcoeff44 * r2 + m->zhcoeff66 * r4 + m->zhcoeff88 * r6 -
                            r3i);
            }
        }
    }
}

/* ForceField::calc_pairwise with the model's electrostatics and HPS (ForceField.cpp:333-418). */
static void calc_pair_f32_m(float *ev, float *ee, double w[3], const float c1[3], const float c2[3], float p6,
                            float p12, float hcut, float hlam, float q1, float q2, double cutoff, const ogo_ele *m,
                            const ogo_hps *h) {
    float d[3];
    for (int k = 0; k < 3; k++) d[k] = c1[k] - c2[k];
    float r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    float r  = sqrtf(r2);
    *ev = *ee = 0.0f;
    w[0] = w[1] = w[2] = 0.0;
    if ((double)r >= cutoff) return;
    float r_inv = (float)(1.0 / (double)r), r2_inv = (float)(1.0 / (double)r2);
    float r3_inv = r_inv * r2_inv, r6_inv = r3_inv * r3_inv, r12_inv = r6_inv * r6_inv;
    float t6 = p6 * r6_inv, t12 = p12 * r12_inv;
    *ev = -t6 + t12;
    float wc = (float)((double)r2_inv * (-12.0 * (double)t12 + 6.0 * (double)t6));
    if (h && h->on) {
        if (r > hcut) {
            *ev *= hlam;
            wc *= hlam;
        } else {
            *ev += (1 - hlam) * h->eps;
        }
    }
    float cc = (float)((double)(q1 * q2) * CHARGE_COEFF);
    float gc;
    ele_pair_f(m, ee, &gc, r, r2, r_inv, r2_inv, r3_inv, cc);
    for (int k = 0; k < 3; k++) w[k] = (double)(wc * d[k] + gc * d[k]);
}

void ogo_pair_allpairs_f32_m(const ogo_pbc *p, int n, const double *crd, const float *charge, const int *atom_type,
                             int n_types, const float *lj6, const float *lj12, const int *nb15off, int max_nb15off,
                             double cutoff, const ogo_ele *m, const ogo_hps *h, double *work, double ene[2]) {
    memset(work, 0, sizeof(double) * 3 * (size_t)n);
    ene[0] = ene[1] = 0.0;
    for (int a1 = 0; a1 < n; a1++) {
        float x1[3] = {(float)crd[a1 * 3], (float)crd[a1 * 3 + 1], (float)crd[a1 * 3 + 2]};
        for (int a2 = 0; a2 < a1; a2++) {
            float x2[3] = {(float)crd[a2 * 3], (float)crd[a2 * 3 + 1], (float)crd[a2 * 3 + 2]};
            int excl = 0;
            for (int k = 0; k < max_nb15off; k++)
                if (nb15off[(size_t)a1 * max_nb15off + k] == a2) excl = 1;
            if (excl) continue;
            int ti = atom_type[a1] * n_types + atom_type[a2];
            for (int d = 0; d < 3; d++) {
                if (x2[d] - x1[d] >= p->L_half[d]) x2[d] -= p->L[d];
                else if (x2[d] - x1[d] <= -p->L_half[d]) x2[d] += p->L[d];
            }
            float ev, ee;
            double w[3];
            calc_pair_f32_m(&ev, &ee, w, x1, x2, lj6[ti], lj12[ti], h && h->on ? h->cut[ti] : 0.0f,
                            h && h->on ? h->lambda[ti] : 1.0f, charge[a1], charge[a2], cutoff, m, h);
            ene[0] += (double)ev;
            ene[1] += (double)ee;
            for (int d = 0; d < 3; d++) {
                work[a1 * 3 + d] += w[d];
                work[a2 * 3 + d] -= w[d];
            }
        }
    }
}

double ogo_excess_f32_m(const ogo_pbc *p, int n_excess, const int *ep, const double *crd, const float *charge,
                        const ogo_ele *m, double *work) {
    double sum = 0.0;
    for (int k = 0; k < n_excess; k++) {
        int i = ep[2 * k], j = ep[2 * k + 1];
        float c1[3] = {(float)crd[i * 3], (float)crd[i * 3 + 1], (float)crd[i * 3 + 2]};
        float c2[3] = {(float)crd[j * 3], (float)crd[j * 3 + 1], (float)crd[j * 3 + 2]};
        float d[3];
        diff_minim_f(p, d, c1, c2);
        /* ForceField::calc_zms_excess (ForceField.cpp:420-437) */
        float r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        float r = sqrtf(r2);
        float ri = (float)(1.0 / (double)r);
        float r2i = ri * ri, r3i = r2i * ri;
        float cc = (float)((double)(charge[i] * charge[j]) * CHARGE_COEFF);
        float e, g;
        ele_excess_f(m, &e, &g, r, r2, ri, r2i, r3i, cc);
        sum += (double)e;
        for (int q = 0; q < 3; q++) {
            double w = (double)(g * d[q]);
            work[i * 3 + q] += w;
            work[j * 3 + q] -= w;
        }
    }
    return sum;
}

double ogo_self_energy_m(int n, int n_excess, const int *ep, const float *charge, const ogo_ele *m) {
    double *dw = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    for (int k = 0; k < n_excess; k++) {
        dw[ep[2 * k]] += (double)charge[ep[2 * k + 1]];
        dw[ep[2 * k + 1]] += (double)charge[ep[2 * k]];
    }
    float mon = 0.0f;
    const double zmcore = (double)m->zmcore;
    for (int i = 0; i < n; i++) {
        const double q = (double)charge[i];
        const double es = ((double)(-m->piewald * charge[i] * charge[i]) - zmcore * q * (q + dw[i])) * 0.5 * CHARGE_COEFF;
        mon = (float)((double)mon + es);
    }
    free(dw);
    return (double)mon;
}

/* FP64 forms of the same functions, for the parity oracle. */
static void ele_pair_d(const ogo_ele64 *m, double *e, double *g, double r, double r2, double cc) {
    const double ri = 1.0 / r, r2i = 1.0 / r2, r3i = ri * r2i, r4 = r2 * r2, r6 = r4 * r2, r8 = r4 * r4;
    if (m->mode == OGO_ELE_DH) {
        *e = cc * ri * m->dielectric_inv * exp(-r * m->debye_length_inv);
        *g = -*e * (ri + m->debye_length_inv);
        return;
    }
    double erc = 1.0, ex = 0.0;
    if (!m->alpha0) {
        const double t = r * m->alpha;
        erc = erfc(t);
        ex = m->piewald * exp(-t * t) * r2i;
    }
    switch (m->mode) {
        case OGO_ELE_ZD:
            *e = cc * (ri * erc - m->zcore + m->bcoeff * r2);
            *g = -cc * (erc * r3i + ex - m->fcoeff);
            break;
        case OGO_ELE_ZQ:
            *e = cc * (ri * erc - m->zqcore - m->zqcoeff2 * r2 - m->zqcoeff4 * r4);
            *g = -cc * (r3i * erc + ex + m->zqcoeff22 + m->zqcoeff44 * r2);
            break;
        case OGO_ELE_ZO:
            *e = cc * (ri * erc - m->zocore - m->zocoeff2 * r2 - m->zocoeff4 * r4 - m->zocoeff6 * r6);
            if (m->alpha0) *g = -cc * (r3i + m->zocoeff22 + m->zocoeff44 * r2 + m->zocoeff66 * r4);
            else *g = -cc * (r3i * erc + ex + m->zhcoeff22 + m->zhcoeff44 * r2 + m->zhcoeff66 * r4);
            break;
        default:
            *e = cc * (ri * erc - m->zhcore - m->zhcoeff2 * r2 - m->zhcoeff4 * r4 - m->zhcoeff6 * r6 - m->zhcoeff8 * r8);
            *g = -cc * (r3i * erc + ex + m->zhcoeff22 + m->zhcoeff44 * r2 + m->zhcoeff66 * r4 + m->zhcoeff88 * r6);
    }
}

static void ele_excess_d(const ogo_ele64 *m, double *e, double *g, double r, double r2, double cc) {
    *e = *g = 0.0;
    if (m->mode == OGO_ELE_DH) return;
    const double ri = 1.0 / r, r2i = ri * ri, r3i = r2i * ri, r4 = r2 * r2, r6 = r4 * r2, r8 = r4 * r4;
    double erc = 1.0, erfn = 0.0, ex = 0.0;
    if (!m->alpha0) {
        const double t = m->alpha * r;
        erc = erfc(t);
        erfn = 1.0 - erc;
        ex = m->piewald * exp(-t * t) * r2i;
    }
    switch (m->mode) {
        case OGO_ELE_ZD:
            if (m->alpha0) {
                *e = cc * m->bcoeff * r2;
                *g = cc * m->fcoeff;
            } else {
                *e = cc * (-erfn * r + m->bcoeff * r2);
                *g = -cc * (erc * r3i + ex - m->fcoeff - r3i);
            }
            break;
        case OGO_ELE_ZQ:
            *e = cc * (-erfn * ri - m->zqcoeff2 * r2 - m->zqcoeff4 * r4);
            *g = -cc * (m->alpha0 ? (m->zqcoeff22 + m->zqcoeff44 * r2)
                                  : (erc * r3i + ex + m->zqcoeff22 + m->zqcoeff44 * r2 - r3i));
            break;
        case OGO_ELE_ZO:
            *e = cc * (-erfn * ri - m->zocoeff2 * r2 - m->zocoeff4 * r4 - m->zocoeff6 * r4 * r);
            *g = -cc * (m->alpha0 ? (m->zocoeff22 + m->zocoeff44 * r2 + m->zocoeff66 * r4)
                                  : (erc * r3i + ex + m->zocoeff22 + m->zocoeff44 * r2 + m->zocoeff66 * r4 - r3i));
            break;
        default:
            if (m->alpha0) {
                *e = cc * (-m->zhcoeff2 * r2 - m->zhcoeff4 * r4 - m->zhcoeff6 * r6 - m->zhcoeff8 * r8);
                *g = -cc * (m->zhcoeff22 + m->zhcoeff44 * r2 + m->zhcoeff66 * r2 + m->zhcoeff88 * r6 - r3i);
            } else {
                *e = cc * (-erfn * ri - m->zhcoeff2 * r2 - m->zhcoeff4 * r4);
                *g = -cc * (erc * r3i + ex + m->zhcoeff22 + m->zhcoeff44 * r2 + m->zhcoeff66 * r4 + m->zhcoeff88 * r6 -
                            r3i);
            }
    }
}

void ogo_pair_cells_f64_m(const double L[3], const ogo_grid *gr, const ogo_cellpairs *cp, const double *crd,
                          const double *charge, const int *atom_type, int n_types, const double *lj6,
                          const double *lj12, double cutoff, const ogo_ele64 *m, const ogo_hps64 *h, double *work,
                          double ene[2], double vir[9]) {
    ene[0] = ene[1] = 0.0;
    for (int k = 0; k < 9; k++) vir[k] = 0.0;
    for (int k = 0; k < cp->n_pairs; k++) {
        int c1 = cp->cell1[k], c2 = cp->cell2[k], img = cp->image[k];
        double sh[3] = {(img & 1) ? -L[0] : (img & 2) ? L[0] : 0.0, (img & 4) ? -L[1] : (img & 8) ? L[1] : 0.0,
                        (img & 16) ? -L[2] : (img & 32) ? L[2] : 0.0};
        for (int a2 = 0; a2 < OGO_N_ATOM_CELL; a2++) {
            int id2 = gr->slot_atomid[c2 * OGO_N_ATOM_CELL + a2];
            for (int a1 = 0; a1 < OGO_N_ATOM_CELL; a1++) {
                if ((cp->mask[k] >> (a2 * OGO_N_ATOM_CELL + a1)) & 1) continue;
                int id1 = gr->slot_atomid[c1 * OGO_N_ATOM_CELL + a1];
                double d[3];
                for (int q = 0; q < 3; q++) d[q] = crd[id1 * 3 + q] - (crd[id2 * 3 + q] + sh[q]);
                double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                if (r2 >= cutoff * cutoff) continue;
                int ti = atom_type[id1] * n_types + atom_type[id2];
                double r = sqrt(r2), r2i = 1.0 / r2, r6i = r2i * r2i * r2i;
                double t6 = lj6[ti] * r6i, t12 = lj12[ti] * r6i * r6i;
                double ev = t12 - t6, wl = r2i * (-12.0 * t12 + 6.0 * t6);
                if (h && h->on) {
                    if (r > h->cut[ti]) {
                        ev *= h->lambda[ti];
                        wl *= h->lambda[ti];
                    } else {
                        ev += (1.0 - h->lambda[ti]) * h->eps;
                    }
                }
                double ee, ge, w[3];
                ele_pair_d(m, &ee, &ge, r, r2, charge[id1] * charge[id2] * CHARGE_COEFF);
                ene[0] += ev;
                ene[1] += ee;
                for (int q = 0; q < 3; q++) {
                    w[q] = (wl + ge) * d[q];
                    work[id1 * 3 + q] += w[q];
                    work[id2 * 3 + q] -= w[q];
                }
                add_vir(vir, d, w);
            }
        }
    }
}

double ogo_excess_f64_m(const double L[3], int n_excess, const int *ep, const double *crd, const double *charge,
                        const ogo_ele64 *m, double *work, double vir[9]) {
    double sum = 0.0;
    for (int k = 0; k < n_excess; k++) {
        int i = ep[2 * k], j = ep[2 * k + 1];
        double d[3], w[3];
        for (int q = 0; q < 3; q++) {
            d[q] = crd[i * 3 + q] - crd[j * 3 + q];
            d[q] -= L[q] * nearbyint(d[q] / L[q]);
        }
        double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        double e, g;
        ele_excess_d(m, &e, &g, sqrt(r2), r2, charge[i] * charge[j] * CHARGE_COEFF);
        sum += e;
        for (int q = 0; q < 3; q++) {
            w[q] = g * d[q];
            work[i * 3 + q] += w[q];
            work[j * 3 + q] -= w[q];
        }
        if (vir) add_vir(vir, d, w);
    }
    return sum;
}
