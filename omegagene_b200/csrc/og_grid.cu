// og_grid.cu -- on-device MiniCell: column assignment, per-column z sort with dummy padding,
// uniform z-grid and the cell-pair list with its 64-bit exclusion masks.
//
// Restates MiniCell::set_atoms_into_grid_xy (src/celeste/core/MiniCell.cpp:292-402, 404-691,
// 785-869), set_uniform_grid (:896-932), enumerate_cell_pairs (:934-1150), check_valid_pair
// (:1152-1162), add_cell_pair (:1163-1203) and set_cell_pair_bitmask (:1204-1237).
// The list comes out in the reference CPU build's order (cell1, then column offset x-major,
// then z image -1/0/+1, then cell2), built count -> scan -> fill, so it is deterministic
// (the reference GPU enumeration appends with atomicAdd, cuda_setup.cu:1007-1012).
//
// This file is compiled with -fmad=false: the float expressions that decide cell membership
// and pair distances must round like the reference's separate multiplies and adds.
#include "og_internal.cuh"

namespace og {

// ---------------------------------------------------------------- columns

// One thread per atom: xy column (MiniCell.cpp:318-345) and the sort key (float z, atom id).
__global__ void k_assign_columns(const SysDev *__restrict__ sys, const int *__restrict__ atom_sys,
                                 const double *__restrict__ crd, int n_atoms,
                                 int *__restrict__ atom_col, unsigned long long *__restrict__ atom_key,
                                 int *__restrict__ col_count, int *__restrict__ counters,
                                 int *__restrict__ sys_fault) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_atoms) return;
    const SysDev &S = sys[atom_sys[a]];
    int c[2];
    bool bad = false;
    for (int d = 0; d < 2; d++) {
        float x = __double2float_rn(crd[3 * a + d] - (double)S.lowerf[d]);
        if (!(fabsf(x) < 64.0f * S.Lf[d])) { bad = true; x = 0.0f; }
        const int nd = d == 0 ? S.nx : S.ny;
        int ci;
        if (x >= 0.0f && x <= S.Lf[d]) {
            // An in-box coordinate stays in the column that holds it.  Within a few
            // microangstroms of the upper face x, or x / L_cell, rounds up to the box length or
            // the column count, which the reference wraps to column 0 (MiniCell.cpp:329-335,
            // :1251-1259): the atom would sit one box length from the grid coordinate it keeps,
            // and its pairs within the cutoff would be missed until the next build.
            ci = min((int)floorf(__fdiv_rn(x, S.L_cell[d])), nd - 1);
        } else {
            for (int it = 0; it < 128 && x < 0.0f; it++) x = __fadd_rn(x, S.Lf[d]);
            for (int it = 0; it < 128 && x >= S.Lf[d]; it++) x = __fsub_rn(x, S.Lf[d]);
            ci = (int)floorf(__fdiv_rn(x, S.L_cell[d]));
            // MiniCell::get_column_id_from_crd (:1251-1259)
            if (ci < 0) ci += nd;
            if (ci >= nd) ci -= nd;
        }
        if (ci < 0 || ci >= nd) { bad = true; ci = 0; }
        c[d] = ci;
    }
    if (bad) {
        og_set_flag(counters, OG_FLAG_BAD_COORD);
        atomicOr(&sys_fault[atom_sys[a]], OG_FLAG_BAD_COORD);
    }
    int col = S.col_base + c[0] + c[1] * S.nx;
    atom_col[a] = col;
    float zf = __double2float_rn(crd[3 * a + 2]);
    atom_key[a] = ((unsigned long long)og_float_order(zf) << 32) | (unsigned int)(a - S.atom_base);
    atomicAdd(&col_count[col], 1);
}

// Single block: exclusive scans over all columns of atom counts and of 8-atom cells
// (MiniCell::set_idx_xy_head, :785-861); empty columns get head -1.
__global__ void k_scan_columns(const int *__restrict__ col_count, int n_cols,
                               int *__restrict__ col_atom_start, int *__restrict__ col_cell_start,
                               int *__restrict__ col_head_cell, int *__restrict__ counters,
                               const int *__restrict__ sys_col_base, int n_sys, int *__restrict__ sys_cell_base) {
    __shared__ int s_a[1024], s_c[1024];
    __shared__ int carry_a, carry_c;
    if (threadIdx.x == 0) { carry_a = 0; carry_c = 0; }
    __syncthreads();
    for (int base = 0; base < n_cols; base += blockDim.x) {
        int i = base + threadIdx.x;
        int na = i < n_cols ? col_count[i] : 0;
        int nc = (na + OG_CELL - 1) / OG_CELL;
        s_a[threadIdx.x] = na;
        s_c[threadIdx.x] = nc;
        __syncthreads();
        for (int off = 1; off < blockDim.x; off <<= 1) {
            int va = threadIdx.x >= off ? s_a[threadIdx.x - off] : 0;
            int vc = threadIdx.x >= off ? s_c[threadIdx.x - off] : 0;
            __syncthreads();
            s_a[threadIdx.x] += va;
            s_c[threadIdx.x] += vc;
            __syncthreads();
        }
        if (i < n_cols) {
            int ea = carry_a + s_a[threadIdx.x] - na;
            int ec = carry_c + s_c[threadIdx.x] - nc;
            col_atom_start[i] = ea;
            col_cell_start[i] = ec;
            col_head_cell[i] = na == 0 ? -1 : ec;
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) {
            carry_a += s_a[threadIdx.x];
            carry_c += s_c[threadIdx.x];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        col_atom_start[n_cols] = carry_a;
        col_cell_start[n_cols] = carry_c;
        counters[OG_CNT_N_CELLS] = carry_c;
        counters[OG_CNT_LIST_BUILDS]++;
    }
    __syncthreads();
    for (int s = threadIdx.x; s <= n_sys; s += blockDim.x)
        sys_cell_base[s] = col_cell_start[sys_col_base[s]];
}

__global__ void k_scatter_columns(const int *__restrict__ atom_col, const unsigned long long *__restrict__ atom_key,
                                  int n_atoms, const int *__restrict__ col_atom_start, int *__restrict__ col_fill,
                                  unsigned long long *__restrict__ col_keys) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_atoms) return;
    int col = atom_col[a];
    int pos = atomicAdd(&col_fill[col], 1);
    col_keys[col_atom_start[col] + pos] = atom_key[a];
}

// One block per column: bitonic sort of (float z, atom id) keys in shared memory, then the
// column's slots (atoms in z order, dummies copying the last atom, MiniCell.cpp:531-613) and
// cells.  Slot coordinates are the float-rounded positions the reference grid holds.
__global__ void k_sort_columns(const int *__restrict__ col_count, const int *__restrict__ col_atom_start,
                               const int *__restrict__ col_cell_start, const int *__restrict__ col_sys,
                               const unsigned long long *__restrict__ col_keys, const SysDev *__restrict__ sys,
                               const double *__restrict__ crd, int *__restrict__ slot_atom,
                               double *__restrict__ slot_crd, int *__restrict__ atom_slot,
                               int *__restrict__ cell_col, int *__restrict__ cell_sys, int *__restrict__ counters,
                               int *__restrict__ sys_fault) {
    __shared__ unsigned long long keys[OG_MAX_COLUMN_ATOMS];
    const int col = blockIdx.x;
    const int n = col_count[col];
    if (n == 0) return;
    const unsigned long long *src = col_keys + col_atom_start[col];
    // A column beyond the sort capacity (a blown-up system piles its atoms into one column) is
    // flagged, which faults the call and undoes it, and still laid out, unsorted, from the
    // keys in global memory: every slot, cell and atom index of the build stays valid for the
    // kernels that run until the call ends.
    const bool over = n > OG_MAX_COLUMN_ATOMS;
    const unsigned long long *K = over ? src : keys;
    if (over) {
        if (threadIdx.x == 0) {
            og_set_flag(counters, OG_FLAG_COLUMN_CAPACITY);
            atomicOr(&sys_fault[col_sys[col]], OG_FLAG_COLUMN_CAPACITY);
        }
    } else {
        int np2 = 1;
        while (np2 < n) np2 <<= 1;
        for (int i = threadIdx.x; i < np2; i += blockDim.x) keys[i] = i < n ? src[i] : ~0ull;
        __syncthreads();
        for (int k = 2; k <= np2; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < np2; i += blockDim.x) {
                    int ixj = i ^ j;
                    if (ixj > i) {
                        unsigned long long a = keys[i], b = keys[ixj];
                        bool up = (i & k) == 0;
                        if ((a > b) == up) { keys[i] = b; keys[ixj] = a; }
                    }
                }
                __syncthreads();
            }
        }
    }
    const int s = col_sys[col];
    const int atom_base = sys[s].atom_base;
    const int head = col_cell_start[col];
    const int ncz = (n + OG_CELL - 1) / OG_CELL;
    for (int k = threadIdx.x; k < ncz * OG_CELL; k += blockDim.x) {
        int use = k < n ? k : n - 1;
        int atom = atom_base + (int)(K[use] & 0xffffffffull);
        int slot = head * OG_CELL + k;
        slot_atom[slot] = k < n ? atom : -1;
        for (int d = 0; d < 3; d++) slot_crd[3 * slot + d] = (double)__double2float_rn(crd[3 * atom + d]);
        if (k < n) atom_slot[atom] = slot;
    }
    for (int k = threadIdx.x; k < ncz; k += blockDim.x) {
        cell_col[head + k] = col;
        cell_sys[head + k] = s;
    }
}

// One thread per cell: origin, float z extent, real-atom byte and the uniform z-grid
// (MiniCell::set_uniform_grid, :896-932).  uni_lo starts at INT_MAX (empty), uni_hi at -1.
__global__ void k_cell_info(const int *__restrict__ counters, int cells_cap, const int *__restrict__ cell_col,
                            const int *__restrict__ cell_sys, const int *__restrict__ col_cell_start,
                            const SysDev *__restrict__ sys, const double *__restrict__ slot_crd,
                            const int *__restrict__ slot_atom, double *__restrict__ cell_origin,
                            float2 *__restrict__ cell_zr, int2 *__restrict__ cell_uni,
                            unsigned char *__restrict__ cell_valid, int *__restrict__ uni_lo,
                            int *__restrict__ uni_hi) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int n_cells = counters[OG_CNT_N_CELLS];
    if (c >= n_cells || c >= cells_cap) return;
    const int col = cell_col[c];
    const SysDev &S = sys[cell_sys[c]];
    const int lcol = col - S.col_base;
    const int cx = lcol % S.nx, cy = lcol / S.nx, cz = c - col_cell_start[col];
    const double *p0 = slot_crd + 3 * (size_t)(c * OG_CELL);
    cell_origin[3 * c + 0] = p0[0];
    cell_origin[3 * c + 1] = p0[1];
    cell_origin[3 * c + 2] = p0[2];
    float zmin = (float)p0[2];
    float zmax = (float)slot_crd[3 * (size_t)(c * OG_CELL + OG_CELL - 1) + 2];
    cell_zr[c] = make_float2(zmin, zmax);
    unsigned v = 0;
    for (int k = 0; k < OG_CELL; k++) v |= (slot_atom[c * OG_CELL + k] >= 0 ? 1u : 0u) << k;
    cell_valid[c] = (unsigned char)v;
    int umin = __float2int_rz(__fdiv_rn(__fsub_rn(zmin, S.lowerf[2]), S.L_z_uni));
    int umax = __float2int_rz(__fdiv_rn(__fsub_rn(zmax, S.lowerf[2]), S.L_z_uni));
    // Bins of the cell's own column.  A cell whose top lies within float rounding of the upper
    // face divides out to bin n_uni_z, which the reference registers as the next column's bin 0
    // (MiniCell.cpp:912-926): no cell of its own column then finds it, and the pairs it should
    // form with them are lost until the next build.  It belongs to bin n_uni_z - 1.  (The clamp
    // also holds a runaway coordinate of a blown-up system, whose call is undone, in range.)
    umin = max(0, min(umin, S.n_uni_z - 1));
    umax = max(0, min(umax, S.n_uni_z - 1));
    cell_uni[c] = make_int2(umin, umax);
    const int n_uni = S.n_columns * S.n_uni_z;
    int steps = 0;
    for (int z = umin; z <= umax && steps <= S.n_uni_z + 1; z++, steps++) {
        int u = cx * S.n_uni_z + cy * (S.n_uni_z * S.nx) + z;
        if (u < 0 || u >= n_uni) continue;
        atomicMin(&uni_lo[S.uni_base + u], cz);
        atomicMax(&uni_hi[S.uni_base + u], cz);
    }
}

// ------------------------------------------------------------- cell pairs

__device__ __forceinline__ bool valid_pair(int c1, int c2) {
    bool o1 = (c1 & 1) != 0, o2 = (c2 & 1) != 0;
    if (o1) return !((c2 < c1 && !o2) || (c2 > c1 && o2));
    return !((c2 < c1 && o2) || (c2 > c1 && !o2));
}

// 64-bit mask of a cell pair: bit a2*8+a1 set = pair skipped (MiniCell.cpp:1204-1237).
// Per cell, once per list build: the excluded partners of its atoms as (partner cell << 6 |
// mask bit) entries, so that the mask of each of the cell's ~100 cell pairs scans one short
// contiguous row instead of chasing atom -> partner -> slot for all 8 atoms.  row[0] = entry
// count, or -1 when the row is full or cell indices do not fit the packing (the mask then takes
// the direct path).
__global__ void k_cell_excl(const int *__restrict__ counters, int cells_cap, const int *__restrict__ slot_atom,
                            const int *__restrict__ atom_slot, const int *__restrict__ excl_start,
                            const int *__restrict__ excl_list, int *__restrict__ cell_excl) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int n_cells = counters[OG_CNT_N_CELLS];
    if (c >= n_cells || c >= cells_cap) return;
    int *row = cell_excl + (size_t)c * OG_CELL_EXCL;
    int n = 0;
    bool full = cells_cap >= (1 << 25);
    for (int i1 = 0; i1 < OG_CELL && !full; i1++) {
        const int a = slot_atom[c * OG_CELL + i1];
        if (a < 0) continue;
        for (int e = excl_start[a]; e < excl_start[a + 1]; e++) {
            const int sl = atom_slot[excl_list[e]];
            if (n + 1 >= OG_CELL_EXCL) { full = true; break; }
            row[1 + n++] = ((sl >> 3) << 6) | ((sl & 7) * 8 + i1);
        }
    }
    row[0] = full ? -1 : n;
}

__device__ __forceinline__ unsigned long long pair_mask(int c1, int c2, unsigned v1, unsigned v2,
                                                        const int *__restrict__ slot_atom,
                                                        const int *__restrict__ atom_slot,
                                                        const int *__restrict__ excl_start,
                                                        const int *__restrict__ excl_list,
                                                        const int *__restrict__ cell_excl) {
    unsigned long long valid = 0;
    for (int i2 = 0; i2 < OG_CELL; i2++)
        if ((v2 >> i2) & 1u) valid |= (unsigned long long)v1 << (8 * i2);
    unsigned long long m = ~valid;
    if (c1 == c2) m |= 0x80c0e0f0f8fcfeffull;  // bits i1 >= i2 of every row i2
    const int *row = cell_excl + (size_t)c1 * OG_CELL_EXCL;
    const int n = row[0];
    if (n >= 0) {
        for (int k = 1; k <= n; k++) {
            const int e = row[k];
            if ((e >> 6) == c2) m |= 1ull << (e & 63);
        }
        return m;
    }
    for (int i1 = 0; i1 < OG_CELL; i1++) {
        int a = slot_atom[c1 * OG_CELL + i1];
        if (a < 0) continue;
        for (int e = excl_start[a]; e < excl_start[a + 1]; e++) {
            int sl = atom_slot[excl_list[e]];
            if ((sl >> 3) == c2) m |= 1ull << ((sl & 7) * 8 + i1);
        }
    }
    return m;
}

// Enumerates the cell pairs of one (cell1, neighbour column) exactly like the reference's
// loop body (MiniCell.cpp:968-1140).  With out_c2img == nullptr it only counts; otherwise it
// writes (cell2, image bits) of each pair, and k_pair_records forms the rest of the record.
__device__ int enumerate_column(int c1, int nb, const SysDev &S, int cell_base,
                                const int *__restrict__ cell_col, const int *__restrict__ col_cell_start,
                                const int *__restrict__ col_head_cell, const float2 *__restrict__ cell_zr,
                                const int2 *__restrict__ cell_uni, const int *__restrict__ uni_lo,
                                const int *__restrict__ uni_hi, int2 *out_c2img, int out_cap) {
    const int nx = S.nx, ny = S.ny, nuz = S.n_uni_z;
    const int wy = 2 * S.n_nb[1] + 1;
    const int dcx = nb / wy - S.n_nb[0];
    const int dcy = nb % wy - S.n_nb[1];
    const int lcol1 = cell_col[c1] - S.col_base;
    const int x1 = lcol1 % nx, y1 = lcol1 / nx;
    int rx = x1 + dcx, ix = 0, x2 = rx;
    if (rx < 0) { ix = -1; x2 = nx + rx; }
    else if (rx >= nx) { ix = 1; x2 = rx - nx; }
    int ry = y1 + dcy, iy = 0, y2 = ry;
    if (ry < 0) { iy = -1; y2 = ny + ry; }
    else if (ry >= ny) { iy = 1; y2 = ry - ny; }
    float dx0 = 0.0f, dx1 = 0.0f;
    if (dcx > 0) dx0 = __fmul_rn((float)(dcx - 1), S.L_cell[0]);
    else if (dcx < 0) dx0 = __fmul_rn((float)(dcx + 1), S.L_cell[0]);
    dx0 = __fmul_rn(dx0, dx0);
    if (dcy > 0) dx1 = __fmul_rn((float)(dcy - 1), S.L_cell[1]);
    else if (dcy < 0) dx1 = __fmul_rn((float)(dcy + 1), S.L_cell[1]);
    dx1 = __fmul_rn(dx1, dx1);
    const float dxy = __fadd_rn(dx0, dx1);
    const int2 u1 = cell_uni[c1];
    int first_u[3], last_u[3];
    int tf = u1.x - 2;
    if (tf < 0) { first_u[0] = nuz + tf; last_u[0] = nuz - 1; tf = 0; }
    else { first_u[0] = -1; last_u[0] = -1; }
    first_u[1] = tf;
    int tl = u1.y + 2;
    if (tl >= nuz) { first_u[2] = 0; last_u[2] = tl - nuz; last_u[1] = nuz - 1; }
    else { first_u[2] = -1; last_u[2] = -1; last_u[1] = tl; }
    const int gcol2 = S.col_base + x2 + y2 * nx;
    const int head2 = col_head_cell[gcol2];
    const float2 z1 = cell_zr[c1];
    const int lc1 = c1 - cell_base;
    const int n_uni = S.n_columns * nuz;
    int n = 0;
    for (int ii = 0; ii < 3; ii++) {
        const int iz = ii - 1;
        if (first_u[ii] < 0) continue;
        int fu = x2 * nuz + y2 * (nuz * nx) + first_u[ii];
        int lu = x2 * nuz + y2 * (nuz * nx) + last_u[ii];
        if (fu < 0 || lu >= n_uni) continue;
        // The window's cells run from its first to its last filled bin.  The reference stops at
        // the first empty bin after a filled one (MiniCell.cpp:1062-1076), so a z gap in column
        // 2 of a bin's height or more (7.5 A in a 44.8 A water box) hides every cell beyond it,
        // pairs within the cutoff included.  Without such a gap both give the same list.
        int f = -1, l = -1;
        for (int u = fu; u <= lu; u++)
            if (uni_lo[S.uni_base + u] != 0x7fffffff) {
                if (f < 0) f = u;
                l = u;
            }
        if (f < 0) continue;
        fu = f;
        lu = l;
        const int lo = uni_lo[S.uni_base + fu], hi = uni_hi[S.uni_base + lu];
        if (lo > hi || head2 < 0) continue;
        // z indices stay inside column 2 (a window that runs past the column's last bin, with
        // few bins per column, reads the next column's bins)
        const int last2 = col_cell_start[gcol2 + 1] - 1;
        const float shz = __fmul_rn((float)iz, S.Lf[2]);
        for (int c2 = head2 + lo; c2 <= head2 + hi && c2 <= last2; c2++) {
            const float2 z2 = cell_zr[c2];
            const float z2t = __fadd_rn(z2.y, shz);
            const float z2b = __fadd_rn(z2.x, shz);
            float dz;
            if (z2t < z1.x) { dz = __fsub_rn(z1.x, z2t); dz = __fmul_rn(dz, dz); }
            else if (z2b > z1.y) { dz = __fsub_rn(z2b, z1.y); dz = __fmul_rn(dz, dz); }
            else dz = 0.0f;
            if (__fadd_rn(dxy, dz) > S.cutoff_pair2) continue;
            if (!valid_pair(lc1, c2 - cell_base)) continue;
            if (out_c2img && n < out_cap) {
                int img = 0;
                if (ix == -1) img |= 1; else if (ix == 1) img |= 2;
                if (iy == -1) img |= 4; else if (iy == 1) img |= 8;
                if (iz == -1) img |= 16; else if (iz == 1) img |= 32;
                out_c2img[n] = make_int2(c2, img);
            }
            n++;
        }
    }
    return n;
}

// One thread per (cell1, neighbour column); nnc = max neighbour columns over systems.
__global__ void k_count_pairs(const int *__restrict__ counters, int cells_cap, int nnc,
                              const int *__restrict__ cell_sys, const int *__restrict__ sys_cell_base,
                              const SysDev *__restrict__ sys, const int *__restrict__ cell_col,
                              const int *__restrict__ col_cell_start, const int *__restrict__ col_head_cell,
                              const float2 *__restrict__ cell_zr, const int2 *__restrict__ cell_uni,
                              const int *__restrict__ uni_lo, const int *__restrict__ uni_hi,
                              const int *__restrict__ sys_fault, int *__restrict__ count) {
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)cells_cap * nnc) return;
    const int c1 = (int)(idx / nnc), nb = (int)(idx % nnc);
    const int n_cells = counters[OG_CNT_N_CELLS];
    int n = 0;
    if (c1 < n_cells) {
        const int s = cell_sys[c1];
        const SysDev &S = sys[s];
        // a system already faulted in this call (its coordinates left the box or piled into one
        // column) gets no pairs: the call is undone, and its list would be all pairs of a column
        if (nb < S.n_nb_cols && sys_fault[s] == 0)
            n = enumerate_column(c1, nb, S, sys_cell_base[s], cell_col, col_cell_start, col_head_cell, cell_zr,
                                 cell_uni, uni_lo, uni_hi, nullptr, 0);
    }
    count[idx] = n;
}

__global__ void k_fill_pairs(int *__restrict__ counters, int cells_cap, int nnc, long long pair_cap,
                             const int *__restrict__ cell_sys, const int *__restrict__ sys_cell_base,
                             const SysDev *__restrict__ sys, const int *__restrict__ cell_col,
                             const int *__restrict__ col_cell_start, const int *__restrict__ col_head_cell,
                             const float2 *__restrict__ cell_zr, const int2 *__restrict__ cell_uni,
                             const int *__restrict__ uni_lo, const int *__restrict__ uni_hi,
                             const int *__restrict__ sys_fault, const long long *__restrict__ offset,
                             int2 *__restrict__ cp_c2img) {
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int n_cells = counters[OG_CNT_N_CELLS];
    if (idx >= (long long)n_cells * nnc) return;
    const int c1 = (int)(idx / nnc), nb = (int)(idx % nnc);
    const int s = cell_sys[c1];
    const SysDev &S = sys[s];
    if (nb >= S.n_nb_cols || sys_fault[s] != 0) return;
    const long long off = offset[idx];
    const int cap = (int)max(0ll, min(pair_cap - off, (long long)1 << 30));
    int n = enumerate_column(c1, nb, S, sys_cell_base[s], cell_col, col_cell_start, col_head_cell, cell_zr, cell_uni,
                             uni_lo, uni_hi, cp_c2img + off, cap);
    if (off + n > pair_cap) og_set_flag(counters, OG_FLAG_PAIR_CAPACITY);
}

// The rest of every record once the enumeration has written (cell2, image): the 64-bit
// exclusion mask (the reference's CellPair::pair_mask) and the pair kernel's record (the shift
// from cell1's origin to cell2's image origin, formed in FP64, and cell2).  One warp per
// cell1, lanes over its records: cell1's exclusion row is read once per warp and the writes
// are coalesced.
__global__ void k_pair_records(const int *__restrict__ counters, long long pair_cap, const int *__restrict__ cell_sys,
                               const SysDev *__restrict__ sys, const int *__restrict__ cp_head,
                               const int2 *__restrict__ cp_c2img, const unsigned char *__restrict__ cell_valid,
                               const int *__restrict__ slot_atom, const int *__restrict__ atom_slot,
                               const int *__restrict__ excl_start, const int *__restrict__ excl_list,
                               const int *__restrict__ cell_excl, const double *__restrict__ cell_origin,
                               unsigned long long *__restrict__ cp_mask, float4 *__restrict__ cp_shift) {
    const int c1 = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (c1 >= counters[OG_CNT_N_CELLS]) return;
    const SysDev &S = sys[cell_sys[c1]];
    const long long k1 = min((long long)cp_head[c1 + 1], pair_cap);
    const unsigned v1 = cell_valid[c1];
    const double o1x = cell_origin[3 * c1], o1y = cell_origin[3 * c1 + 1], o1z = cell_origin[3 * c1 + 2];
    for (long long k = (long long)cp_head[c1] + lane; k < k1; k += 32) {
        const int2 ci = cp_c2img[k];
        const int c2 = ci.x, img = ci.y;
        cp_mask[k] = pair_mask(c1, c2, v1, cell_valid[c2], slot_atom, atom_slot, excl_start, excl_list, cell_excl);
        const double shx = (img & 1) ? -S.L[0] : ((img & 2) ? S.L[0] : 0.0);
        const double shy = (img & 4) ? -S.L[1] : ((img & 8) ? S.L[1] : 0.0);
        const double shz = (img & 16) ? -S.L[2] : ((img & 32) ? S.L[2] : 0.0);
        cp_shift[k] = make_float4((float)(cell_origin[3 * c2] + shx - o1x), (float)(cell_origin[3 * c2 + 1] + shy - o1y),
                                  (float)(cell_origin[3 * c2 + 2] + shz - o1z), __int_as_float(c2));
    }
}

// CSR heads from the scanned counts; also publishes the total.
// Heads are held within the buffer (pair_cap): past it the list is incomplete, the fill flags
// it, and every kernel that walks [cp_head[c], cp_head[c + 1]) stays inside the buffer.
__global__ void k_pair_heads(int *__restrict__ counters, int cells_cap, int nnc, long long pair_cap,
                             const long long *__restrict__ offset, int *__restrict__ cp_head) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int n_cells = counters[OG_CNT_N_CELLS];
    const long long total = offset[(long long)cells_cap * nnc];
    if (c > cells_cap) return;
    cp_head[c] = (int)min(c < n_cells ? offset[(long long)c * nnc] : total, pair_cap);
    if (c == 0) counters[OG_CNT_N_PAIRS] = (int)min(total, 2147483647ll);
}

// ------------------------------------------------------------------ scan

// Exclusive scan of an int array in blocks of 2*blockDim (Blelloch-free Hillis-Steele per
// block, then block totals are scanned by the same kernel recursively from the host).
// 64-bit sums: the pair counts of a blown-up system (its atoms piled into one column) can total
// more than 2^31, and a wrapped offset would send the list fill outside its buffer.
template <typename TI>
__global__ void k_scan_block(const TI *__restrict__ in, long long *__restrict__ out, long long n,
                             long long *__restrict__ block_sums) {
    __shared__ long long s[2048];
    const long long base = (long long)blockIdx.x * 2048;
    for (int k = 0; k < 2; k++) {
        long long i = base + threadIdx.x + k * 1024;
        s[threadIdx.x + k * 1024] = i < n ? in[i] : 0;
    }
    __syncthreads();
    // up-sweep / down-sweep (work-efficient) over 2048 elements
    int off = 1;
    for (int d = 1024; d > 0; d >>= 1) {
        __syncthreads();
        if (threadIdx.x < d) {
            int ai = off * (2 * threadIdx.x + 1) - 1;
            int bi = off * (2 * threadIdx.x + 2) - 1;
            s[bi] += s[ai];
        }
        off <<= 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (block_sums) block_sums[blockIdx.x] = s[2047];
        s[2047] = 0;
    }
    for (int d = 1; d < 2048; d <<= 1) {
        off >>= 1;
        __syncthreads();
        if (threadIdx.x < d) {
            int ai = off * (2 * threadIdx.x + 1) - 1;
            int bi = off * (2 * threadIdx.x + 2) - 1;
            long long t = s[ai];
            s[ai] = s[bi];
            s[bi] += t;
        }
    }
    __syncthreads();
    for (int k = 0; k < 2; k++) {
        long long i = base + threadIdx.x + k * 1024;
        if (i < n) out[i] = s[threadIdx.x + k * 1024];
    }
}
template __global__ void k_scan_block<int>(const int *, long long *, long long, long long *);
template __global__ void k_scan_block<long long>(const long long *, long long *, long long, long long *);

__global__ void k_scan_add(long long *__restrict__ out, long long n, const long long *__restrict__ block_offsets) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += block_offsets[i / 2048];
}

}  // namespace og
