// og_pair.cu -- Lennard-Jones + zero-dipole (alpha = 0) pair forces over the cell-pair list.
//
// Physics of ForceField::calc_pairwise + ZeroMultipoleSum::calc_zero02pole_alpha0
// (src/celeste/core/ForceField.cpp:333-418, ZeroMultipoleSum.cpp:309-332) and the reference
// GPU kernel kernel_pairwise_ljzd / cal_pair (src/celeste/cuda/cuda_setup.cu:487-675):
//   E_vdw = C12/r^12 - C6/r^6
//   E_ele = q_i q_j 332.06378 (1/r - zcore + bcoeff r^2),  r < cutoff
//   dE/dx_i = [r^-2 (6 C6/r^6 - 12 C12/r^12) - cc (r^-3 - fcoeff)] (x_i - x_j)
//
// B200 layout: one warp per cell1; lane = (i-group g = lane>>3, j-slot jj = lane&7); each lane
// evaluates i = g and i = g+4 against j = jj of every cell2 in cell1's CSR range.
// Coordinates are float offsets from a per-cell FP64 origin, and each cell pair carries the
// float shift origin2 + image - origin1 formed in FP64 when the list was built, so a pair
// distance carries the rounding of a ~10 A quantity instead of an absolute coordinate.
// A warp-uniform test on per-step cell bounding boxes skips cell pairs that are entirely
// beyond the cutoff (the list itself is the reference's 13 A slab list, unchanged).
// Work on j is reduced over the 4 i-groups with shuffles and added to an int64 fixed-point
// accumulator (2^-32 kcal/mol/A), which makes per-atom sums independent of launch order;
// i-work and energies are summed in FP32 over at most 16 cell pairs and then folded into FP64
// registers; energies and the virial go to per-cell slots reduced later in a fixed order.
#include "og_internal.cuh"

namespace og {

// Per-cell bounding box of the real atoms (cell-relative coordinates), refreshed every step.
__global__ void k_cell_bbox(const int *__restrict__ counters, int cells_cap, const float4 *__restrict__ xq,
                            const unsigned char *__restrict__ cell_valid, float4 *__restrict__ bbox) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int n_cells = counters[OG_CNT_N_CELLS];
    if (c >= n_cells || c >= cells_cap) return;
    const unsigned v = cell_valid[c];
    float lx = 3e38f, ly = 3e38f, lz = 3e38f, hx = -3e38f, hy = -3e38f, hz = -3e38f;
    for (int k = 0; k < OG_CELL; k++) {
        if (!((v >> k) & 1u)) continue;
        const float4 p = xq[c * OG_CELL + k];
        lx = fminf(lx, p.x);
        ly = fminf(ly, p.y);
        lz = fminf(lz, p.z);
        hx = fmaxf(hx, p.x);
        hy = fmaxf(hy, p.y);
        hz = fmaxf(hz, p.z);
    }
    bbox[2 * c] = make_float4(lx, ly, lz, 0.f);
    bbox[2 * c + 1] = make_float4(hx, hy, hz, 0.f);
}

#define OG_FLUSH 16
#define OG_FOLD 1  // j-major kernels: rounds (a lane's 8 pairs of one cell pair) per FP64 fold of energies

// MINB = minimum resident blocks per SM the register allocation must allow (2: ~100 registers,
// 3: 80, 4: 64 with a few spills); the engine's autotuner times the variants on the first list.
template <bool VIR, int MINB>
__global__ void __launch_bounds__(256, MINB)
k_pair_ljzd(const int *__restrict__ counters, const int *__restrict__ cell_sys, const SysDev *__restrict__ sys,
            const float4 *__restrict__ bbox, const float4 *__restrict__ xq, const int *__restrict__ slot_type,
            const int *__restrict__ cp_head, const float4 *__restrict__ cp_shift, const int2 *__restrict__ cp_c2img,
            const unsigned long long *__restrict__ cp_mask, const float2 *__restrict__ lj,
            unsigned long long *__restrict__ frc, double *__restrict__ cell_acc, long long pair_cap) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int n_cells = counters[OG_CNT_N_CELLS];
    if (warp >= n_cells) return;
    const int c1 = warp;
    const int jj = lane & 7, g = lane >> 3;
    const SysDev &S = sys[cell_sys[c1]];
    const float4 xi0 = xq[c1 * OG_CELL + g], xi1 = xq[c1 * OG_CELL + g + 4];
    const int ti0 = slot_type[c1 * OG_CELL + g] * S.n_types + S.lj_base;
    const int ti1 = slot_type[c1 * OG_CELL + g + 4] * S.n_types + S.lj_base;
    const float qc0 = xi0.w * (float)OG_CHARGE_COEFF, qc1 = xi1.w * (float)OG_CHARGE_COEFF;
    const float rc2 = S.cutoff2, zcore = S.zcore, bco = S.bcoeff, fco = S.fcoeff;
    // skip threshold with a margin for the float rounding of boxes and shifts
    const float rskip = sqrtf(rc2) + 1e-3f, rskip2 = rskip * rskip;
    const float4 b1l = bbox[2 * c1], b1h = bbox[2 * c1 + 1];
    // FP64 accumulators of this warp's cell1 in shared memory: work of its 8 atoms and the two
    // energies; FP32 partials in registers are folded in every OG_FLUSH cell pairs
    __shared__ double s_acc[8][OG_CELL * 3 + 2];
    double *acc_w = s_acc[(threadIdx.x >> 5) & 7];
    if (lane < OG_CELL * 3 + 2) acc_w[lane] = 0.0;
    __syncwarp();
    float a0x = 0.f, a0y = 0.f, a0z = 0.f, a1x = 0.f, a1y = 0.f, a1z = 0.f, av = 0.f, ae = 0.f;
    int n_acc = 0;
    auto flush = [&]() {
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            a0x += __shfl_xor_sync(0xffffffffu, a0x, o);
            a0y += __shfl_xor_sync(0xffffffffu, a0y, o);
            a0z += __shfl_xor_sync(0xffffffffu, a0z, o);
            a1x += __shfl_xor_sync(0xffffffffu, a1x, o);
            a1y += __shfl_xor_sync(0xffffffffu, a1y, o);
            a1z += __shfl_xor_sync(0xffffffffu, a1z, o);
        }
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            av += __shfl_xor_sync(0xffffffffu, av, o);
            ae += __shfl_xor_sync(0xffffffffu, ae, o);
        }
        if (jj == 0) {
            acc_w[3 * g + 0] += a0x;
            acc_w[3 * g + 1] += a0y;
            acc_w[3 * g + 2] += a0z;
            acc_w[3 * (g + 4) + 0] += a1x;
            acc_w[3 * (g + 4) + 1] += a1y;
            acc_w[3 * (g + 4) + 2] += a1z;
        }
        if (lane == 0) {
            acc_w[OG_CELL * 3] += av;
            acc_w[OG_CELL * 3 + 1] += ae;
        }
        a0x = a0y = a0z = a1x = a1y = a1z = av = ae = 0.f;
        n_acc = 0;
    };
    int n_act = 0;  // interacting pairs (VIR mode only)
    double v[9];
    if (VIR)
        for (int q = 0; q < 9; q++) v[q] = 0;
    // a list that overflowed its buffer is flagged and redone; never read past the buffer
    const int k_beg = cp_head[c1];
    const int k_end = (int)min((long long)cp_head[c1 + 1], pair_cap);
    for (int chunk = k_beg; chunk < k_end; chunk += 32) {
        // each lane fetches one cell-pair record and tests its bounding boxes; the warp then
        // walks the surviving pairs with the next pair's j atom prefetched
        const int kk = chunk + lane;
        float4 my_sp = make_float4(0.f, 0.f, 0.f, 0.f);
        unsigned long long my_m = ~0ull;
        int my_img = 0;
        bool keep = false;
        if (kk < k_end) {
            my_sp = cp_shift[kk];
            const int c2 = __float_as_int(my_sp.w);
            const float4 l2 = bbox[2 * c2], h2 = bbox[2 * c2 + 1];
            const float gx = fmaxf(0.f, fmaxf(l2.x + my_sp.x - b1h.x, b1l.x - (h2.x + my_sp.x)));
            const float gy = fmaxf(0.f, fmaxf(l2.y + my_sp.y - b1h.y, b1l.y - (h2.y + my_sp.y)));
            const float gz = fmaxf(0.f, fmaxf(l2.z + my_sp.z - b1h.z, b1l.z - (h2.z + my_sp.z)));
            keep = gx * gx + gy * gy + gz * gz < rskip2;
            if (keep) my_m = cp_mask[kk];
            if (VIR && keep) my_img = cp_c2img[kk].y;
        }
        unsigned ballot = __ballot_sync(0xffffffffu, keep);
        if (!ballot) continue;
        int src = __ffs(ballot) - 1;
        ballot &= ballot - 1;
        float4 sp;
        sp.x = __shfl_sync(0xffffffffu, my_sp.x, src);
        sp.y = __shfl_sync(0xffffffffu, my_sp.y, src);
        sp.z = __shfl_sync(0xffffffffu, my_sp.z, src);
        sp.w = __shfl_sync(0xffffffffu, my_sp.w, src);
        int c2 = __float_as_int(sp.w);
        float4 xj = xq[c2 * OG_CELL + jj];
        int tj = slot_type[c2 * OG_CELL + jj];
        while (true) {
            const unsigned long long m = __shfl_sync(0xffffffffu, my_m, src);
            const int img = VIR ? __shfl_sync(0xffffffffu, my_img, src) : 0;
            const int cur_c2 = c2;
            const float4 cur_sp = sp, cur_xj = xj;
            const int cur_tj = tj;
            const bool more = ballot != 0;
            if (more) {  // prefetch the next surviving pair
                src = __ffs(ballot) - 1;
                ballot &= ballot - 1;
                sp.x = __shfl_sync(0xffffffffu, my_sp.x, src);
                sp.y = __shfl_sync(0xffffffffu, my_sp.y, src);
                sp.z = __shfl_sync(0xffffffffu, my_sp.z, src);
                sp.w = __shfl_sync(0xffffffffu, my_sp.w, src);
                c2 = __float_as_int(sp.w);
                xj = xq[c2 * OG_CELL + jj];
                tj = slot_type[c2 * OG_CELL + jj];
            }
            const float rjx = cur_xj.x + cur_sp.x, rjy = cur_xj.y + cur_sp.y, rjz = cur_xj.z + cur_sp.z;
            float wjx = 0.f, wjy = 0.f, wjz = 0.f;
#pragma unroll
            for (int t = 0; t < 2; t++) {
                const float4 xi = t ? xi1 : xi0;
                const float dx = xi.x - rjx, dy = xi.y - rjy, dz = xi.z - rjz;
                const float r2 = dx * dx + dy * dy + dz * dz;
                const int bit = jj * OG_CELL + g + 4 * t;
                const bool act = (((m >> bit) & 1ull) == 0ull) && (r2 < rc2);
                const float r2s = act ? r2 : 1.0f;
                // hardware estimate + one Newton step on the exact residual 1 - r2 y^2 (FMA):
                // the estimate alone carries a one-sided error that adds up over millions of
                // Coulomb pairs in the energy
                float rinv = rsqrtf(r2s);
                const float hres = fmaf(-r2s * rinv, rinv, 1.0f);
                rinv = fmaf(0.5f * rinv, hres, rinv);
                const float r2inv = rinv * rinv;
                const float r6inv = r2inv * r2inv * r2inv;
                const float2 p = __ldg(&lj[(t ? ti1 : ti0) + cur_tj]);
                const float t6 = p.x * r6inv, t12 = p.y * r6inv * r6inv;
                const float cc = (t ? qc1 : qc0) * cur_xj.w;
                float pv = t12 - t6;
                float pe = cc * (rinv - zcore + bco * r2s);
                float wc = r2inv * (6.0f * t6 - 12.0f * t12) - cc * (rinv * r2inv - fco);
                if (!act) { pv = 0.f; pe = 0.f; wc = 0.f; }
                if (VIR) n_act += act ? 1 : 0;
                const float wx = wc * dx, wy = wc * dy, wz = wc * dz;
                av += pv;
                ae += pe;
                wjx -= wx;
                wjy -= wy;
                wjz -= wz;
                if (t) { a1x += wx; a1y += wy; a1z += wz; }
                else { a0x += wx; a0y += wy; a0z += wz; }
            }
            if (++n_acc == OG_FLUSH) flush();
            // work on j: sum over the four i-groups (lanes jj, jj+8, jj+16, jj+24)
            wjx += __shfl_xor_sync(0xffffffffu, wjx, 8);
            wjy += __shfl_xor_sync(0xffffffffu, wjy, 8);
            wjz += __shfl_xor_sync(0xffffffffu, wjz, 8);
            wjx += __shfl_xor_sync(0xffffffffu, wjx, 16);
            wjy += __shfl_xor_sync(0xffffffffu, wjy, 16);
            wjz += __shfl_xor_sync(0xffffffffu, wjz, 16);
            if (g == 0 && (wjx != 0.f || wjy != 0.f || wjz != 0.f)) {
                unsigned long long *fj = frc + 3 * (size_t)(cur_c2 * OG_CELL + jj);
                atomicAdd(fj + 0, (unsigned long long)__float2ll_rn(wjx * (float)OG_FIX_SCALE));
                atomicAdd(fj + 1, (unsigned long long)__float2ll_rn(wjy * (float)OG_FIX_SCALE));
                atomicAdd(fj + 2, (unsigned long long)__float2ll_rn(wjz * (float)OG_FIX_SCALE));
                if (VIR && img != 0) {
                    // sum over pairs of d (x) f = sum_atoms x (x) F + sum_cell-pairs shift (x) F_j
                    const double sh[3] = {(img & 1) ? -S.L[0] : ((img & 2) ? S.L[0] : 0.0),
                                          (img & 4) ? -S.L[1] : ((img & 8) ? S.L[1] : 0.0),
                                          (img & 16) ? -S.L[2] : ((img & 32) ? S.L[2] : 0.0)};
                    const double fjv[3] = {-(double)wjx, -(double)wjy, -(double)wjz};
                    for (int a = 0; a < 3; a++)
                        for (int b = 0; b < 3; b++) v[a * 3 + b] += sh[a] * fjv[b];
                }
            }
            if (!more) break;
        }
    }
    flush();
    __syncwarp();
    // work on i: one fixed-point add per component of each of the 8 atoms
    if (lane < OG_CELL) {
        const double wx = acc_w[3 * lane], wy = acc_w[3 * lane + 1], wz = acc_w[3 * lane + 2];
        if (wx != 0.0 || wy != 0.0 || wz != 0.0) {
            unsigned long long *fa = frc + 3 * (size_t)(c1 * OG_CELL + lane);
            atomicAdd(fa + 0, (unsigned long long)og_to_fix(wx));
            atomicAdd(fa + 1, (unsigned long long)og_to_fix(wy));
            atomicAdd(fa + 2, (unsigned long long)og_to_fix(wz));
        }
    }
    const double e_vdw = acc_w[OG_CELL * 3], e_ele = acc_w[OG_CELL * 3 + 1];
    if (VIR) {
        for (int q = 0; q < 9; q++)
            for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
        for (int o = 16; o > 0; o >>= 1) n_act += __shfl_xor_sync(0xffffffffu, n_act, o);
    }
    if (lane == 0) {
        double *acc = cell_acc + (size_t)c1 * OG_CELL_ACC;
        acc[0] = e_vdw;
        acc[1] = e_ele;
        if (VIR) {
            for (int q = 0; q < 9; q++) acc[2 + q] = v[q];
            acc[11] = (double)n_act;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// j-major variant: one warp per cell1, four cell pairs at a time (8-lane group q = lane>>3 per
// cell pair, lane jj = lane&7 holds j atom jj of that cell2) and every lane evaluates all 8 i
// atoms against its j.  Per cell pair a lane then does 8 evaluations for one record fetch, one
// j load and one fixed-point add per component (the warp-per-8x8 layout above does 2 and needs
// a 4-lane shuffle reduction of the j work).  The i work stays in 24 FP32 registers per lane
// over that lane's cell pairs (about a quarter of cell1's list) and is reduced across the warp
// in FP64 at the end, in a fixed order.  i atoms are read from shared memory (broadcast).
template <bool VIR, int MINB>
__global__ void __launch_bounds__(256, MINB)
k_pair_ljzd_jm(const int *__restrict__ counters, const int *__restrict__ cell_sys, const SysDev *__restrict__ sys,
               const float4 *__restrict__ bbox, const float4 *__restrict__ xq, const int *__restrict__ slot_type,
               const int *__restrict__ cp_head, const float4 *__restrict__ cp_shift, const int2 *__restrict__ cp_c2img,
               const unsigned long long *__restrict__ cp_mask, const float2 *__restrict__ lj,
               unsigned long long *__restrict__ frc, double *__restrict__ cell_acc, long long pair_cap) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int wib = (threadIdx.x >> 5) & 7;
    const int n_cells = counters[OG_CNT_N_CELLS];
    if (warp >= n_cells) return;
    const int c1 = warp;
    const int jj = lane & 7, q = lane >> 3;
    const SysDev &S = sys[cell_sys[c1]];
    __shared__ float4 s_xi[8][OG_CELL];  // (x, y, z, q * 332.06378) of cell1's atoms, per warp
    __shared__ int s_ti[8][OG_CELL];     // LJ table row of each cell1 atom
    if (lane < OG_CELL) {
        float4 x = xq[c1 * OG_CELL + lane];
        x.w *= (float)OG_CHARGE_COEFF;
        s_xi[wib][lane] = x;
        s_ti[wib][lane] = slot_type[c1 * OG_CELL + lane] * S.n_types + S.lj_base;
    }
    __syncwarp();
    const float rc2 = S.cutoff2, zcore = S.zcore, bco = S.bcoeff, fco = S.fcoeff;
    const float rskip = sqrtf(rc2) + 1e-3f, rskip2 = rskip * rskip;
    const float4 b1l = bbox[2 * c1], b1h = bbox[2 * c1 + 1];
    float fi[OG_CELL][3];
#pragma unroll
    for (int i = 0; i < OG_CELL; i++) fi[i][0] = fi[i][1] = fi[i][2] = 0.f;
    float av = 0.f, ae = 0.f;     // FP32 energy partials of up to OG_FOLD rounds ...
    double dv = 0.0, de = 0.0;    // ... folded into FP64
    int n_round = 0;
    int n_act = 0;
    double v[9];
    if (VIR)
        for (int k = 0; k < 9; k++) v[k] = 0;
    const int k_beg = cp_head[c1];
    const int k_end = (int)min((long long)cp_head[c1 + 1], pair_cap);
    for (int chunk = k_beg; chunk < k_end; chunk += 32) {
        // one record per lane, bounding-box test, then the survivors four at a time
        const int kk = chunk + lane;
        float4 my_sp = make_float4(0.f, 0.f, 0.f, 0.f);
        unsigned long long my_m = ~0ull;
        int my_img = 0;
        bool keep = false;
        if (kk < k_end) {
            my_sp = cp_shift[kk];
            const int c2 = __float_as_int(my_sp.w);
            const float4 l2 = bbox[2 * c2], h2 = bbox[2 * c2 + 1];
            const float gx = fmaxf(0.f, fmaxf(l2.x + my_sp.x - b1h.x, b1l.x - (h2.x + my_sp.x)));
            const float gy = fmaxf(0.f, fmaxf(l2.y + my_sp.y - b1h.y, b1l.y - (h2.y + my_sp.y)));
            const float gz = fmaxf(0.f, fmaxf(l2.z + my_sp.z - b1h.z, b1l.z - (h2.z + my_sp.z)));
            keep = gx * gx + gy * gy + gz * gz < rskip2;
            if (keep) my_m = cp_mask[kk];
            if (VIR && keep) my_img = cp_c2img[kk].y;
        }
        const unsigned ballot = __ballot_sync(0xffffffffu, keep);
        const int n_keep = __popc(ballot);
        for (int r = 0; r < n_keep; r += 4) {
            const int idx = r + q;
            const bool active = idx < n_keep;
            const int src = active ? (int)__fns(ballot, 0, idx + 1) : 0;
            float4 sp;
            sp.x = __shfl_sync(0xffffffffu, my_sp.x, src);
            sp.y = __shfl_sync(0xffffffffu, my_sp.y, src);
            sp.z = __shfl_sync(0xffffffffu, my_sp.z, src);
            sp.w = __shfl_sync(0xffffffffu, my_sp.w, src);
            const unsigned long long m = __shfl_sync(0xffffffffu, my_m, src);
            const int img = VIR ? __shfl_sync(0xffffffffu, my_img, src) : 0;
            const int c2 = __float_as_int(sp.w);
            float4 xj = make_float4(0.f, 0.f, 0.f, 0.f);
            int tj = 0;
            if (active) {
                xj = xq[c2 * OG_CELL + jj];
                tj = slot_type[c2 * OG_CELL + jj];
            }
            // bits jj*8 + i of the mask: excluded pairs and dummy slots of this j
            const unsigned skip = active ? (unsigned)(m >> (jj * OG_CELL)) & 0xffu : 0xffu;
            const float rjx = xj.x + sp.x, rjy = xj.y + sp.y, rjz = xj.z + sp.z;
            float wjx = 0.f, wjy = 0.f, wjz = 0.f;
#pragma unroll
            for (int i = 0; i < OG_CELL; i++) {
                const float4 xi = s_xi[wib][i];
                const float dx = xi.x - rjx, dy = xi.y - rjy, dz = xi.z - rjz;
                const float r2 = dx * dx + dy * dy + dz * dz;
                const bool act = ((skip >> i) & 1u) == 0u && r2 < rc2;
                const float r2s = act ? r2 : 1.0f;
                float rinv = rsqrtf(r2s);
                const float hres = fmaf(-r2s * rinv, rinv, 1.0f);
                rinv = fmaf(0.5f * rinv, hres, rinv);
                const float r2inv = rinv * rinv;
                const float r6inv = r2inv * r2inv * r2inv;
                const float2 p = __ldg(&lj[s_ti[wib][i] + tj]);
                const float t6 = p.x * r6inv, t12 = p.y * r6inv * r6inv;
                const float cc = xi.w * xj.w;
                float pv = t12 - t6;
                float pe = cc * (rinv - zcore + bco * r2s);
                float wc = r2inv * (6.0f * t6 - 12.0f * t12) - cc * (rinv * r2inv - fco);
                if (!act) { pv = 0.f; pe = 0.f; wc = 0.f; }
                if (VIR) n_act += act ? 1 : 0;
                const float wx = wc * dx, wy = wc * dy, wz = wc * dz;
                av += pv;
                ae += pe;
                fi[i][0] += wx;
                fi[i][1] += wy;
                fi[i][2] += wz;
                wjx -= wx;
                wjy -= wy;
                wjz -= wz;
            }
            if (++n_round == OG_FOLD) {
                dv += (double)av;
                de += (double)ae;
                av = ae = 0.f;
                n_round = 0;
            }
            if (active && (wjx != 0.f || wjy != 0.f || wjz != 0.f)) {
                unsigned long long *fj = frc + 3 * (size_t)(c2 * OG_CELL + jj);
                atomicAdd(fj + 0, (unsigned long long)__float2ll_rn(wjx * (float)OG_FIX_SCALE));
                atomicAdd(fj + 1, (unsigned long long)__float2ll_rn(wjy * (float)OG_FIX_SCALE));
                atomicAdd(fj + 2, (unsigned long long)__float2ll_rn(wjz * (float)OG_FIX_SCALE));
                if (VIR && img != 0) {
                    const double sh[3] = {(img & 1) ? -S.L[0] : ((img & 2) ? S.L[0] : 0.0),
                                          (img & 4) ? -S.L[1] : ((img & 8) ? S.L[1] : 0.0),
                                          (img & 16) ? -S.L[2] : ((img & 32) ? S.L[2] : 0.0)};
                    const double fjv[3] = {-(double)wjx, -(double)wjy, -(double)wjz};
                    for (int a = 0; a < 3; a++)
                        for (int b = 0; b < 3; b++) v[a * 3 + b] += sh[a] * fjv[b];
                }
            }
        }
    }
    // i work: FP64 butterfly over the 32 lanes (fixed order), then one fixed-point add per
    // component of each of the 8 atoms
    double mine[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < OG_CELL; i++) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            double x = (double)fi[i][d];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if (lane == i) mine[d] = x;
        }
    }
    if (lane < OG_CELL && (mine[0] != 0.0 || mine[1] != 0.0 || mine[2] != 0.0)) {
        unsigned long long *fa = frc + 3 * (size_t)(c1 * OG_CELL + lane);
        atomicAdd(fa + 0, (unsigned long long)og_to_fix(mine[0]));
        atomicAdd(fa + 1, (unsigned long long)og_to_fix(mine[1]));
        atomicAdd(fa + 2, (unsigned long long)og_to_fix(mine[2]));
    }
    double e_vdw = dv + (double)av, e_ele = de + (double)ae;
    for (int o = 16; o > 0; o >>= 1) {
        e_vdw += __shfl_xor_sync(0xffffffffu, e_vdw, o);
        e_ele += __shfl_xor_sync(0xffffffffu, e_ele, o);
    }
    if (VIR) {
        for (int k = 0; k < 9; k++)
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
        for (int o = 16; o > 0; o >>= 1) n_act += __shfl_xor_sync(0xffffffffu, n_act, o);
    }
    if (lane == 0) {
        double *acc = cell_acc + (size_t)c1 * OG_CELL_ACC;
        acc[0] = e_vdw;
        acc[1] = e_ele;
        if (VIR) {
            for (int k = 0; k < 9; k++) acc[2 + k] = v[k];
            acc[11] = (double)n_act;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// j-major with sm_100 packed FP32 (FFMA2 / FADD2 / FMUL2): the 8 i atoms are taken two at a
// time, so one instruction advances the arithmetic of both pairs (i = 2p and 2p+1) of a lane.
// Only the reciprocal square root, the cutoff / mask tests and the table loads stay scalar.
// The arithmetic per pair, and its rounding, is that of the scalar kernels (each component of
// __ffma2_rn rounds like __fmaf_rn); only the order in which partial sums are added differs.
__device__ __forceinline__ float2 og_f2(float a, float b) { return make_float2(a, b); }

// ENE = false skips the energies (pair terms, their sums and the per-cell energy slots): the
// step path asks for them only on the steps whose energies are read.
template <bool VIR, bool ENE, int MINB>
__global__ void __launch_bounds__(256, MINB)
k_pair_ljzd_jm2(const int *__restrict__ counters, const int *__restrict__ cell_sys, const SysDev *__restrict__ sys,
                const float4 *__restrict__ bbox, const float4 *__restrict__ xq, const int *__restrict__ slot_type,
                const int *__restrict__ cp_head, const float4 *__restrict__ cp_shift, const int2 *__restrict__ cp_c2img,
                const unsigned long long *__restrict__ cp_mask, const float2 *__restrict__ lj,
                unsigned long long *__restrict__ frc, double *__restrict__ cell_acc, long long pair_cap) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int wib = (threadIdx.x >> 5) & 7;
    const int n_cells = counters[OG_CNT_N_CELLS];
    if (warp >= n_cells) return;
    const int c1 = warp;
    const int jj = lane & 7, q = lane >> 3;
    const SysDev &S = sys[cell_sys[c1]];
    // per warp, i atoms in pairs p = (2p, 2p+1): {x_a, x_b, y_a, y_b}, {z_a, z_b, qc_a, qc_b}
    __shared__ float4 s_ab[8][OG_CELL / 2][2];
    __shared__ int2 s_t2[8][OG_CELL / 2];
    if (lane < OG_CELL / 2) {
        const float4 a = xq[c1 * OG_CELL + 2 * lane], b = xq[c1 * OG_CELL + 2 * lane + 1];
        s_ab[wib][lane][0] = make_float4(a.x, b.x, a.y, b.y);
        s_ab[wib][lane][1] = make_float4(a.z, b.z, a.w * (float)OG_CHARGE_COEFF, b.w * (float)OG_CHARGE_COEFF);
        s_t2[wib][lane] = make_int2(slot_type[c1 * OG_CELL + 2 * lane] * S.n_types + S.lj_base,
                                    slot_type[c1 * OG_CELL + 2 * lane + 1] * S.n_types + S.lj_base);
    }
    __syncwarp();
    const float rc2 = S.cutoff2;
    const float2 nzcore = og_f2(-S.zcore, -S.zcore), bco = og_f2(S.bcoeff, S.bcoeff);
    const float2 nfco = og_f2(-S.fcoeff, -S.fcoeff);
    const float2 one = og_f2(1.f, 1.f), half = og_f2(0.5f, 0.5f), six = og_f2(6.f, 6.f);
    const float2 m12 = og_f2(-12.f, -12.f), mone = og_f2(-1.f, -1.f);
    const float rskip = sqrtf(rc2) + 1e-3f, rskip2 = rskip * rskip;
    const float4 b1l = bbox[2 * c1], b1h = bbox[2 * c1 + 1];
    float2 fx[OG_CELL / 2], fy[OG_CELL / 2], fz[OG_CELL / 2];
#pragma unroll
    for (int p = 0; p < OG_CELL / 2; p++) fx[p] = fy[p] = fz[p] = og_f2(0.f, 0.f);
    float2 av = og_f2(0.f, 0.f), ae = og_f2(0.f, 0.f);  // FP32 partials of up to OG_FOLD rounds ...
    double dv = 0.0, de = 0.0;                          // ... folded into FP64
    int n_round = 0;
    int n_act = 0;
    double v[9];
    if (VIR)
        for (int k = 0; k < 9; k++) v[k] = 0;
    const int k_beg = cp_head[c1];
    const int k_end = (int)min((long long)cp_head[c1 + 1], pair_cap);
    for (int chunk = k_beg; chunk < k_end; chunk += 32) {
        const int kk = chunk + lane;
        float4 my_sp = make_float4(0.f, 0.f, 0.f, 0.f);
        unsigned long long my_m = ~0ull;
        int my_img = 0;
        bool keep = false;
        if (kk < k_end) {
            my_sp = cp_shift[kk];
            const int c2 = __float_as_int(my_sp.w);
            const float4 l2 = bbox[2 * c2], h2 = bbox[2 * c2 + 1];
            const float gx = fmaxf(0.f, fmaxf(l2.x + my_sp.x - b1h.x, b1l.x - (h2.x + my_sp.x)));
            const float gy = fmaxf(0.f, fmaxf(l2.y + my_sp.y - b1h.y, b1l.y - (h2.y + my_sp.y)));
            const float gz = fmaxf(0.f, fmaxf(l2.z + my_sp.z - b1h.z, b1l.z - (h2.z + my_sp.z)));
            keep = gx * gx + gy * gy + gz * gz < rskip2;
            if (keep) my_m = cp_mask[kk];
            if (VIR && keep) my_img = cp_c2img[kk].y;
        }
        const unsigned ballot = __ballot_sync(0xffffffffu, keep);
        const int n_keep = __popc(ballot);
        for (int r = 0; r < n_keep; r += 4) {
            const int idx = r + q;
            const bool active = idx < n_keep;
            const int src = active ? (int)__fns(ballot, 0, idx + 1) : 0;
            float4 sp;
            sp.x = __shfl_sync(0xffffffffu, my_sp.x, src);
            sp.y = __shfl_sync(0xffffffffu, my_sp.y, src);
            sp.z = __shfl_sync(0xffffffffu, my_sp.z, src);
            sp.w = __shfl_sync(0xffffffffu, my_sp.w, src);
            const unsigned long long m = __shfl_sync(0xffffffffu, my_m, src);
            const int img = VIR ? __shfl_sync(0xffffffffu, my_img, src) : 0;
            const int c2 = __float_as_int(sp.w);
            float4 xj = make_float4(0.f, 0.f, 0.f, 0.f);
            int tj = 0;
            if (active) {
                xj = xq[c2 * OG_CELL + jj];
                tj = slot_type[c2 * OG_CELL + jj];
            }
            const unsigned skip = active ? (unsigned)(m >> (jj * OG_CELL)) & 0xffu : 0xffu;
            const float rjx = xj.x + sp.x, rjy = xj.y + sp.y, rjz = xj.z + sp.z;
            const float2 nrx = og_f2(-rjx, -rjx), nry = og_f2(-rjy, -rjy), nrz = og_f2(-rjz, -rjz);
            const float2 qj = og_f2(xj.w, xj.w);
            float2 wjx = og_f2(0.f, 0.f), wjy = og_f2(0.f, 0.f), wjz = og_f2(0.f, 0.f);
#pragma unroll
            for (int p = 0; p < OG_CELL / 2; p++) {
                const float4 A = s_ab[wib][p][0], B = s_ab[wib][p][1];
                const int2 T = s_t2[wib][p];
                const float2 dx = __fadd2_rn(og_f2(A.x, A.y), nrx);
                const float2 dy = __fadd2_rn(og_f2(A.z, A.w), nry);
                const float2 dz = __fadd2_rn(og_f2(B.x, B.y), nrz);
                const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
                const bool act_a = ((skip >> (2 * p)) & 1u) == 0u && r2.x < rc2;
                const bool act_b = ((skip >> (2 * p + 1)) & 1u) == 0u && r2.y < rc2;
                const float2 r2s = og_f2(act_a ? r2.x : 1.0f, act_b ? r2.y : 1.0f);
                float2 y = og_f2(rsqrtf(r2s.x), rsqrtf(r2s.y));
                // one Newton step on the exact residual 1 - r2 y^2, as in the scalar kernels
                const float2 h = __ffma2_rn(__fmul2_rn(__fmul2_rn(r2s, mone), y), y, one);
                y = __ffma2_rn(__fmul2_rn(half, y), h, y);
                const float2 r2inv = __fmul2_rn(y, y);
                const float2 r6 = __fmul2_rn(__fmul2_rn(r2inv, r2inv), r2inv);
                const float2 pa = __ldg(&lj[T.x + tj]), pb = __ldg(&lj[T.y + tj]);
                const float2 t6 = __fmul2_rn(og_f2(pa.x, pb.x), r6);
                const float2 t12 = __fmul2_rn(__fmul2_rn(og_f2(pa.y, pb.y), r6), r6);
                const float2 cc = __fmul2_rn(og_f2(B.z, B.w), qj);
                float2 pv = __ffma2_rn(t6, mone, t12);
                float2 pe = __fmul2_rn(cc, __ffma2_rn(bco, r2s, __fadd2_rn(y, nzcore)));
                // r2^-1 (6 t6 - 12 t12) - cc (r^-3 - fcoeff)
                float2 wc = __ffma2_rn(__fmul2_rn(cc, mone), __ffma2_rn(y, r2inv, nfco),
                                       __fmul2_rn(r2inv, __ffma2_rn(t12, m12, __fmul2_rn(six, t6))));
                const float2 on = og_f2(act_a ? 1.f : 0.f, act_b ? 1.f : 0.f);
                pv = __fmul2_rn(pv, on);
                pe = __fmul2_rn(pe, on);
                wc = __fmul2_rn(wc, on);
                if (VIR) n_act += (act_a ? 1 : 0) + (act_b ? 1 : 0);
                const float2 wx = __fmul2_rn(wc, dx), wy = __fmul2_rn(wc, dy), wz = __fmul2_rn(wc, dz);
                if (ENE) {
                    av = __fadd2_rn(av, pv);
                    ae = __fadd2_rn(ae, pe);
                }
                fx[p] = __fadd2_rn(fx[p], wx);
                fy[p] = __fadd2_rn(fy[p], wy);
                fz[p] = __fadd2_rn(fz[p], wz);
                wjx = __fadd2_rn(wjx, wx);
                wjy = __fadd2_rn(wjy, wy);
                wjz = __fadd2_rn(wjz, wz);
            }
            if (ENE && ++n_round == OG_FOLD) {
                dv += (double)av.x + (double)av.y;
                de += (double)ae.x + (double)ae.y;
                av = ae = og_f2(0.f, 0.f);
                n_round = 0;
            }
            const float sx = -(wjx.x + wjx.y), sy = -(wjy.x + wjy.y), sz = -(wjz.x + wjz.y);
            if (active && (sx != 0.f || sy != 0.f || sz != 0.f)) {
                unsigned long long *fj = frc + 3 * (size_t)(c2 * OG_CELL + jj);
                atomicAdd(fj + 0, (unsigned long long)__float2ll_rn(sx * (float)OG_FIX_SCALE));
                atomicAdd(fj + 1, (unsigned long long)__float2ll_rn(sy * (float)OG_FIX_SCALE));
                atomicAdd(fj + 2, (unsigned long long)__float2ll_rn(sz * (float)OG_FIX_SCALE));
                if (VIR && img != 0) {
                    const double sh[3] = {(img & 1) ? -S.L[0] : ((img & 2) ? S.L[0] : 0.0),
                                          (img & 4) ? -S.L[1] : ((img & 8) ? S.L[1] : 0.0),
                                          (img & 16) ? -S.L[2] : ((img & 32) ? S.L[2] : 0.0)};
                    // sum over pairs of d (x) f: f on i is +w, so the shift term takes -(work on j)
                    const double fjv[3] = {-(double)sx, -(double)sy, -(double)sz};
                    for (int a = 0; a < 3; a++)
                        for (int b = 0; b < 3; b++) v[a * 3 + b] += sh[a] * fjv[b];
                }
            }
        }
    }
    double mine[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int p = 0; p < OG_CELL / 2; p++) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            double w3[3] = {(double)(h ? fx[p].y : fx[p].x), (double)(h ? fy[p].y : fy[p].x),
                            (double)(h ? fz[p].y : fz[p].x)};
#pragma unroll
            for (int d = 0; d < 3; d++) {
                double x = w3[d];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                if (lane == 2 * p + h) mine[d] = x;
            }
        }
    }
    if (lane < OG_CELL && (mine[0] != 0.0 || mine[1] != 0.0 || mine[2] != 0.0)) {
        unsigned long long *fa = frc + 3 * (size_t)(c1 * OG_CELL + lane);
        atomicAdd(fa + 0, (unsigned long long)og_to_fix(mine[0]));
        atomicAdd(fa + 1, (unsigned long long)og_to_fix(mine[1]));
        atomicAdd(fa + 2, (unsigned long long)og_to_fix(mine[2]));
    }
    if (!ENE) return;
    double e_vdw = dv + (double)av.x + (double)av.y, e_ele = de + (double)ae.x + (double)ae.y;
    for (int o = 16; o > 0; o >>= 1) {
        e_vdw += __shfl_xor_sync(0xffffffffu, e_vdw, o);
        e_ele += __shfl_xor_sync(0xffffffffu, e_ele, o);
    }
    if (VIR) {
        for (int k = 0; k < 9; k++)
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
        for (int o = 16; o > 0; o >>= 1) n_act += __shfl_xor_sync(0xffffffffu, n_act, o);
    }
    if (lane == 0) {
        double *acc = cell_acc + (size_t)c1 * OG_CELL_ACC;
        acc[0] = e_vdw;
        acc[1] = e_ele;
        if (VIR) {
            for (int k = 0; k < 9; k++) acc[2 + k] = v[k];
            acc[11] = (double)n_act;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// j-queue: the packed j-major kernel with a second cull at the j-atom level.  Per warp, the
// surviving cell pairs are expanded four at a time into their 8 j atoms; a j atom farther than
// the cutoff from cell1's bounding box cannot interact with any i atom and is dropped, the rest
// go into a per-warp ring of 64 entries in shared memory (j position relative to cell1's
// frame, charge, type, slot, mask byte).  Whenever 32 entries are waiting, every lane takes one
// and evaluates it against the 8 i atoms.  On water about 40% of the j atoms of a surviving cell
// pair drop out, and every evaluation round runs with all 32 lanes busy.
#define OG_JQ 64

// The electrostatics of one pair for models other than zero-dipole alpha = 0
// (ZeroMultipoleSum.cpp:309-455 and calc_debye_huckel): energy e and gradient coefficient g
// (work = g d), in FP32 with CUDA's erfcf / expf where alpha > 0.  The octupole alpha > 0
// gradient takes the hexadecapole coefficients, as the reference's does.
__device__ __forceinline__ void og_ele_pair(const EleDev &E, float r, float r2, float ri, float r2i, float r3i,
                                            float cc, float &e, float &g) {
    if (E.mode == OG_ELE_DH) {
        const float ld = expf(-r * E.debye_inv);
        e = cc * ri * E.dielectric_inv * ld;
        g = -e * (ri + E.debye_inv);
        return;
    }
    float erc = 1.f, ex = 0.f;
    if (!E.alpha0) {
        const float t = r * E.alpha;
        erc = erfcf(t);
        ex = E.piewald * expf(-t * t) * r2i;
    }
    const float r4 = r2 * r2, r6 = r4 * r2, r8 = r4 * r4;
    switch (E.mode) {
        case OG_ELE_ZD:
            e = cc * (ri * erc - E.zcore + E.bcoeff * r2);
            g = -cc * (erc * r3i + ex - E.fcoeff);
            break;
        case OG_ELE_ZQ:
            e = cc * (ri * erc - E.zqcore - E.zq2 * r2 - E.zq4 * r4);
            g = -cc * (r3i * erc + ex + E.zq22 + E.zq44 * r2);
            break;
        case OG_ELE_ZO:
            e = cc * (ri * erc - E.zocore - E.zo2 * r2 - E.zo4 * r4 - E.zo6 * r6);
            g = E.alpha0 ? -cc * (r3i + E.zo22 + E.zo44 * r2 + E.zo66 * r4)
                         : -cc * (r3i * erc + ex + E.zh22 + E.zh44 * r2 + E.zh66 * r4);
            break;
        default:
            e = cc * (ri * erc - E.zhcore - E.zh2 * r2 - E.zh4 * r4 - E.zh6 * r6 - E.zh8 * r8);
            g = -cc * (r3i * erc + ex + E.zh22 + E.zh44 * r2 + E.zh66 * r4 + E.zh88 * r6);
    }
}

// Per-lane partial sums of one warp's i cell in the j-queue and j-list kernels: i forces of the
// packed pair slots (2p, 2p+1), energies folded into FP64 after every evaluation round, and the
// virial terms.
template <bool VIR>
struct OgIAcc {
    float2 fx[OG_CELL / 2], fy[OG_CELL / 2], fz[OG_CELL / 2];
    double dv, de;
    int n_act;
    double v[VIR ? 9 : 1];
};

template <bool VIR>
__device__ __forceinline__ void og_iacc_zero(OgIAcc<VIR> &A) {
#pragma unroll
    for (int p = 0; p < OG_CELL / 2; p++) A.fx[p] = A.fy[p] = A.fz[p] = og_f2(0.f, 0.f);
    A.dv = A.de = 0.0;
    A.n_act = 0;
#pragma unroll
    for (int k = 0; k < (VIR ? 9 : 1); k++) A.v[k] = 0.0;
}

// A warp's i cell in shared memory: positions and scaled charges packed by pair (2p, 2p+1), and
// the LJ-table row offsets of the atoms' types.
struct OgICell {
    float4 ab[OG_CELL / 2][2];
    int2 t2[OG_CELL / 2];
};

// GEN = false: the row offsets point into the force-scaled copy of the LJ table (6 C6, 12 C12).
template <bool GEN>
__device__ __forceinline__ void og_load_icell(OgICell &ic, int c1, int lane, const float4 *__restrict__ xq,
                                              const int *__restrict__ slot_type, const SysDev &S) {
    if (lane < OG_CELL / 2) {
        const float4 a = xq[c1 * OG_CELL + 2 * lane], b = xq[c1 * OG_CELL + 2 * lane + 1];
        const int base = S.lj_base + (GEN ? 0 : S.ljf_off);
        ic.ab[lane][0] = make_float4(a.x, b.x, a.y, b.y);
        ic.ab[lane][1] = make_float4(a.z, b.z, a.w * (float)OG_CHARGE_COEFF, b.w * (float)OG_CHARGE_COEFF);
        ic.t2[lane] = make_int2(slot_type[c1 * OG_CELL + 2 * lane] * S.n_types + base,
                                slot_type[c1 * OG_CELL + 2 * lane + 1] * S.n_types + base);
    }
    __syncwarp();
}

// The zero-dipole constants of a system, packed for both halves of a pair.
struct OgZdConst {
    float rc2;
    float2 nzcore, bco, nfco;
};

__device__ __forceinline__ OgZdConst og_zd_const(const SysDev &S) {
    OgZdConst k;
    k.rc2 = S.cutoff2;
    k.nzcore = og_f2(-S.zcore, -S.zcore);
    k.bco = og_f2(S.bcoeff, S.bcoeff);
    k.nfco = og_f2(-S.fcoeff, -S.fcoeff);
    return k;
}

// One lane evaluates one j atom against the warp's 8 i atoms: xj is the j position in cell1's
// frame with its charge in w, tj its LJ type, skip its exclusion byte over the i atoms (bit i
// set: no pair), slot its force slot and img the image bits of its cell pair (virial shift term).
// i work goes to the lane's partial sums, j work to the fixed-point accumulator; a lane with
// active = false evaluates a dummy entry whose pairs are all skipped.
// GEN: the system's EleDev model and HPS table (ele, hps) instead of the packed zero-dipole
// alpha = 0 evaluation; both halves of a packed pair are evaluated one after the other.
template <bool VIR, bool ENE, bool GEN>
__device__ __forceinline__ void og_eval_j(OgIAcc<VIR> &A, bool active, float4 xj, int tj, unsigned skip, int slot,
                                          int img, const OgICell &ic, const OgZdConst &K, const SysDev &S,
                                          const EleDev &E, const float2 *__restrict__ lj,
                                          const float2 *__restrict__ hps, unsigned long long *__restrict__ frc) {
    const float2 one = og_f2(1.f, 1.f), half = og_f2(0.5f, 0.5f), mone = og_f2(-1.f, -1.f);
    const float2 nrx = og_f2(-xj.x, -xj.x), nry = og_f2(-xj.y, -xj.y), nrz = og_f2(-xj.z, -xj.z);
    // GEN: +q_j; zero-dipole path: -q_j, so cc below is -q_i q_j (the sign the work takes)
    const float2 qj = GEN ? og_f2(xj.w, xj.w) : og_f2(-xj.w, -xj.w);
    float2 av = og_f2(0.f, 0.f), ae = og_f2(0.f, 0.f);
    float2 wjx = og_f2(0.f, 0.f), wjy = og_f2(0.f, 0.f), wjz = og_f2(0.f, 0.f);
#pragma unroll
    for (int p = 0; p < OG_CELL / 2; p++) {
        const float4 Ap = ic.ab[p][0], Bp = ic.ab[p][1];
        const int2 T = ic.t2[p];
        const float2 dx = __fadd2_rn(og_f2(Ap.x, Ap.y), nrx);
        const float2 dy = __fadd2_rn(og_f2(Ap.z, Ap.w), nry);
        const float2 dz = __fadd2_rn(og_f2(Bp.x, Bp.y), nrz);
        const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
        const bool act_a = ((skip >> (2 * p)) & 1u) == 0u && r2.x < K.rc2;
        const bool act_b = ((skip >> (2 * p + 1)) & 1u) == 0u && r2.y < K.rc2;
        // zero-dipole path: a skipped pair takes r2 = +inf, so rsqrt gives 0 and every inverse
        // power vanishes; with the ZD force constant masked too its work is 0 without a 0/1
        // multiply.  rsqrtf alone (2 ulp) is the inverse distance of the forces: well inside
        // their 1e-5 bar, and a central force of r alone, so still conservative.  The generic
        // path keeps one Newton step and the 0/1 mask.
        const float2 r2s = GEN ? og_f2(act_a ? r2.x : 1.0f, act_b ? r2.y : 1.0f)
                               : og_f2(act_a ? r2.x : __int_as_float(0x7f800000), act_b ? r2.y : __int_as_float(0x7f800000));
        float2 y = og_f2(rsqrtf(r2s.x), rsqrtf(r2s.y));
        if (GEN) {
            const float2 h = __ffma2_rn(__fmul2_rn(__fmul2_rn(r2s, mone), y), y, one);
            y = __ffma2_rn(__fmul2_rn(half, y), h, y);
        }
        const float2 r2inv = __fmul2_rn(y, y);
        const float2 r6 = __fmul2_rn(__fmul2_rn(r2inv, r2inv), r2inv);
        const float2 pa = __ldg(&lj[T.x + tj]), pb = __ldg(&lj[T.y + tj]);
        const float2 c6p = og_f2(pa.x, pb.x), c12p = og_f2(pa.y, pb.y);
        // zero-dipole path: t6 = 6 C6 / r^6 and t12 = 12 C12 / r^12 from the scaled table
        const float2 t6 = __fmul2_rn(c6p, r6);
        const float2 t12 = __fmul2_rn(__fmul2_rn(c12p, r6), r6);
        const float2 cc = __fmul2_rn(og_f2(Bp.z, Bp.w), qj);
        const float2 on = og_f2(act_a ? 1.f : 0.f, act_b ? 1.f : 0.f);
        float2 wc;
        if (!GEN) {
            // work = -q_i q_j (1/r^3 - fco) + (6 C6/r^6 - 12 C12/r^12) / r^2, cc = -q_i q_j
            const float2 nfco = og_f2(act_a ? K.nfco.x : 0.f, act_b ? K.nfco.y : 0.f);
            wc = __ffma2_rn(cc, __ffma2_rn(y, r2inv, nfco), __fmul2_rn(r2inv, __ffma2_rn(t12, mone, t6)));
            if (ENE) {
                // the Ele energy is a small net of large pair terms of both signs: its 1/r takes
                // the Newton step (the forces above do not, so a step's forces are the same
                // whether or not it reports energies).  The energies of skipped pairs (r2s = +inf,
                // ye = NaN) are masked explicitly
                const float2 ye = __ffma2_rn(__fmul2_rn(half, y), __ffma2_rn(__fmul2_rn(__fmul2_rn(r2s, mone), y), y, one), y);
                const float2 pv = __ffma2_rn(t12, og_f2(1.f / 12.f, 1.f / 12.f), __fmul2_rn(t6, og_f2(-1.f / 6.f, -1.f / 6.f)));
                const float2 pe = __fmul2_rn(cc, __ffma2_rn(K.bco, r2s, __fadd2_rn(ye, K.nzcore)));
                av = __fadd2_rn(av, pv);
                ae = __fadd2_rn(ae, og_f2(act_a ? -pe.x : 0.f, act_b ? -pe.y : 0.f));
            }
        } else {
            float w2[2], v2[2], e2[2];
#pragma unroll
            for (int hh = 0; hh < 2; hh++) {
                const float r2h = hh ? r2s.y : r2s.x, yh = hh ? y.y : y.x;
                const float r2i = yh * yh, r3i = yh * r2i, rr = r2h * yh;
                const float t6h = hh ? t6.y : t6.x, t12h = hh ? t12.y : t12.x;
                float ev = t12h - t6h, wl = r2i * (6.f * t6h - 12.f * t12h);
                if (E.hps) {  // ForceField.cpp:380-391
                    const float2 hp = __ldg(&hps[(hh ? T.y : T.x) + tj]);
                    if (rr > hp.x) {
                        ev *= hp.y;
                        wl *= hp.y;
                    } else {
                        ev += (1.f - hp.y) * E.hps_eps;
                    }
                }
                float ee, ge;
                og_ele_pair(E, rr, r2h, yh, r2i, r3i, hh ? cc.y : cc.x, ee, ge);
                w2[hh] = wl + ge;
                v2[hh] = ev;
                e2[hh] = ee;
            }
            wc = __fmul2_rn(og_f2(w2[0], w2[1]), on);
            if (ENE) {
                av = __fadd2_rn(av, __fmul2_rn(og_f2(v2[0], v2[1]), on));
                ae = __fadd2_rn(ae, __fmul2_rn(og_f2(e2[0], e2[1]), on));
            }
        }
        if (VIR) A.n_act += (act_a ? 1 : 0) + (act_b ? 1 : 0);
        A.fx[p] = __ffma2_rn(wc, dx, A.fx[p]);
        A.fy[p] = __ffma2_rn(wc, dy, A.fy[p]);
        A.fz[p] = __ffma2_rn(wc, dz, A.fz[p]);
        wjx = __ffma2_rn(wc, dx, wjx);
        wjy = __ffma2_rn(wc, dy, wjy);
        wjz = __ffma2_rn(wc, dz, wjz);
    }
    if (ENE) {
        A.dv += (double)av.x + (double)av.y;
        A.de += (double)ae.x + (double)ae.y;
    }
    const float sx = -(wjx.x + wjx.y), sy = -(wjy.x + wjy.y), sz = -(wjz.x + wjz.y);
    if (active && (sx != 0.f || sy != 0.f || sz != 0.f)) {
        unsigned long long *fj = frc + 3 * (size_t)slot;
        atomicAdd(fj + 0, (unsigned long long)__float2ll_rn(sx * (float)OG_FIX_SCALE));
        atomicAdd(fj + 1, (unsigned long long)__float2ll_rn(sy * (float)OG_FIX_SCALE));
        atomicAdd(fj + 2, (unsigned long long)__float2ll_rn(sz * (float)OG_FIX_SCALE));
        if (VIR && img != 0) {
            const double sh[3] = {(img & 1) ? -S.L[0] : ((img & 2) ? S.L[0] : 0.0),
                                  (img & 4) ? -S.L[1] : ((img & 8) ? S.L[1] : 0.0),
                                  (img & 16) ? -S.L[2] : ((img & 32) ? S.L[2] : 0.0)};
            // sum over pairs of d (x) f: f on i is +w, so the shift term takes -(work on j)
            const double fjv[3] = {-(double)sx, -(double)sy, -(double)sz};
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) A.v[a * 3 + b] += sh[a] * fjv[b];
        }
    }
}

// End of a warp's i cell: the lanes' i work reduced in FP64 (fixed shuffle order) and added to
// the fixed-point accumulator; energies, virial and the active-pair count to the cell's slots.
template <bool VIR, bool ENE>
__device__ __forceinline__ void og_flush_icell(OgIAcc<VIR> &A, int c1, int lane, unsigned long long *__restrict__ frc,
                                               double *__restrict__ cell_acc) {
    double mine[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int p = 0; p < OG_CELL / 2; p++) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            double w3[3] = {(double)(h ? A.fx[p].y : A.fx[p].x), (double)(h ? A.fy[p].y : A.fy[p].x),
                            (double)(h ? A.fz[p].y : A.fz[p].x)};
#pragma unroll
            for (int d = 0; d < 3; d++) {
                double x = w3[d];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                if (lane == 2 * p + h) mine[d] = x;
            }
        }
    }
    if (lane < OG_CELL && (mine[0] != 0.0 || mine[1] != 0.0 || mine[2] != 0.0)) {
        unsigned long long *fa = frc + 3 * (size_t)(c1 * OG_CELL + lane);
        atomicAdd(fa + 0, (unsigned long long)og_to_fix(mine[0]));
        atomicAdd(fa + 1, (unsigned long long)og_to_fix(mine[1]));
        atomicAdd(fa + 2, (unsigned long long)og_to_fix(mine[2]));
    }
    if (!ENE) return;
    double e_vdw = A.dv, e_ele = A.de;
    for (int o = 16; o > 0; o >>= 1) {
        e_vdw += __shfl_xor_sync(0xffffffffu, e_vdw, o);
        e_ele += __shfl_xor_sync(0xffffffffu, e_ele, o);
    }
    int n_act = A.n_act;
    if (VIR) {
        for (int k = 0; k < 9; k++)
            for (int o = 16; o > 0; o >>= 1) A.v[k] += __shfl_xor_sync(0xffffffffu, A.v[k], o);
        for (int o = 16; o > 0; o >>= 1) n_act += __shfl_xor_sync(0xffffffffu, n_act, o);
    }
    if (lane == 0) {
        double *acc = cell_acc + (size_t)c1 * OG_CELL_ACC;
        acc[0] = e_vdw;
        acc[1] = e_ele;
        if (VIR) {
            for (int k = 0; k < 9; k++) acc[2 + k] = A.v[k];
            acc[11] = (double)n_act;
        }
    }
}

template <bool VIR, bool ENE, int MINB, int NT = 256, bool GEN = false>
__global__ void __launch_bounds__(NT, MINB)
k_pair_ljzd_jq(const int *__restrict__ counters, const int *__restrict__ cell_sys, const SysDev *__restrict__ sys,
               const float4 *__restrict__ bbox, const float4 *__restrict__ xq, const int *__restrict__ slot_type,
               const int *__restrict__ cp_head, const float4 *__restrict__ cp_shift, const int2 *__restrict__ cp_c2img,
               const unsigned long long *__restrict__ cp_mask, const float2 *__restrict__ lj,
               unsigned long long *__restrict__ frc, double *__restrict__ cell_acc, long long pair_cap,
               const EleDev *__restrict__ ele, const float2 *__restrict__ hps) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int n_cells = counters[OG_CNT_N_CELLS];
    if (warp >= n_cells) return;
    const int c1 = warp;
    const int jj = lane & 7, q = lane >> 3;
    const SysDev &S = sys[cell_sys[c1]];
    const EleDev &E = ele[GEN ? cell_sys[c1] : 0];
    __shared__ OgICell s_i[NT / 32];
    __shared__ float4 s_qx[NT / 32][OG_JQ];  // queued j: (x, y, z) in cell1's frame, charge
    __shared__ int4 s_qi[NT / 32][OG_JQ];    // queued j: LJ type, slot, mask byte, image bits
    __shared__ float4 s_rsp[NT / 32][32];    // surviving records of the current chunk, in order:
    __shared__ uint2 s_rm[NT / 32][32];      //   shift + cell2, exclusion mask,
    __shared__ int s_rimg[NT / 32][VIR ? 32 : 1];  //   image bits (virial only)
    og_load_icell<GEN>(s_i[wib], c1, lane, xq, slot_type, S);
    const OgZdConst K = og_zd_const(S);
    const float rskip = sqrtf(K.rc2) + 1e-3f, rskip2 = rskip * rskip;
    const float4 b1l = bbox[2 * c1], b1h = bbox[2 * c1 + 1];
    OgIAcc<VIR> A;
    og_iacc_zero(A);
    int q_head = 0, q_len = 0;  // ring of queued j entries (warp-uniform)

    // lane takes queue entry (q_head + lane) if lane < n_take and evaluates it against cell1
    auto drain = [&](int n_take) {
        const bool active = lane < n_take;
        const int e = (q_head + lane) & (OG_JQ - 1);
        float4 xj = make_float4(0.f, 0.f, 0.f, 0.f);
        int4 ji = make_int4(0, 0, 0xff, 0);
        if (active) {
            xj = s_qx[wib][e];
            ji = s_qi[wib][e];
        }
        og_eval_j<VIR, ENE, GEN>(A, active, xj, ji.x, (unsigned)ji.z, ji.y, ji.w, s_i[wib], K, S, E, lj, hps, frc);
        __syncwarp();
        q_head = (q_head + n_take) & (OG_JQ - 1);
        q_len -= n_take;
    };

    const int k_beg = cp_head[c1];
    const int k_end = (int)min((long long)cp_head[c1 + 1], pair_cap);
    // each lane's record of the next chunk is loaded one chunk ahead
    float4 nx_sp = make_float4(0.f, 0.f, 0.f, 0.f);
    unsigned long long nx_m = ~0ull;
    int nx_img = 0;
    if (k_beg + lane < k_end) {
        nx_sp = cp_shift[k_beg + lane];
        nx_m = cp_mask[k_beg + lane];
        if (VIR) nx_img = cp_c2img[k_beg + lane].y;
    }
    for (int chunk = k_beg; chunk < k_end; chunk += 32) {
        const int kk = chunk + lane;
        const float4 my_sp = nx_sp;
        const unsigned long long my_m = nx_m;
        const int my_img = nx_img;
        if (kk + 32 < k_end) {
            nx_sp = cp_shift[kk + 32];
            nx_m = cp_mask[kk + 32];
            if (VIR) nx_img = cp_c2img[kk + 32].y;
        }
        bool keep = false;
        if (kk < k_end) {
            const int c2 = __float_as_int(my_sp.w);
            const float4 l2 = bbox[2 * c2], h2 = bbox[2 * c2 + 1];
            const float gx = fmaxf(0.f, fmaxf(l2.x + my_sp.x - b1h.x, b1l.x - (h2.x + my_sp.x)));
            const float gy = fmaxf(0.f, fmaxf(l2.y + my_sp.y - b1h.y, b1l.y - (h2.y + my_sp.y)));
            const float gz = fmaxf(0.f, fmaxf(l2.z + my_sp.z - b1h.z, b1l.z - (h2.z + my_sp.z)));
            keep = gx * gx + gy * gy + gz * gz < rskip2;
        }
        const unsigned ballot = __ballot_sync(0xffffffffu, keep);
        const int n_keep = __popc(ballot);
        if (keep) {  // compact the survivors in list order
            const int rank = __popc(ballot & ((1u << lane) - 1u));
            s_rsp[wib][rank] = my_sp;
            s_rm[wib][rank] = make_uint2((unsigned)my_m, (unsigned)(my_m >> 32));
            if (VIR) s_rimg[wib][rank] = my_img;
        }
        __syncwarp();
        for (int r = 0; r < n_keep; r += 4) {
            // expand four surviving cell pairs into their j atoms; queue those near cell1
            const int idx = r + q;
            const bool active = idx < n_keep;
            float4 sp = make_float4(0.f, 0.f, 0.f, 0.f);
            unsigned long long m = ~0ull;
            int img = 0;
            if (active) {
                sp = s_rsp[wib][idx];
                const uint2 mm = s_rm[wib][idx];
                m = ((unsigned long long)mm.y << 32) | mm.x;
                if (VIR) img = s_rimg[wib][idx];
            }
            const int c2 = __float_as_int(sp.w);
            bool push = false;
            float4 xj = make_float4(0.f, 0.f, 0.f, 0.f);
            int tj = 0;
            const unsigned skip = active ? (unsigned)(m >> (jj * OG_CELL)) & 0xffu : 0xffu;
            if (active && skip != 0xffu) {
                xj = xq[c2 * OG_CELL + jj];
                tj = slot_type[c2 * OG_CELL + jj];
                xj.x += sp.x;
                xj.y += sp.y;
                xj.z += sp.z;
                const float gx = fmaxf(0.f, fmaxf(xj.x - b1h.x, b1l.x - xj.x));
                const float gy = fmaxf(0.f, fmaxf(xj.y - b1h.y, b1l.y - xj.y));
                const float gz = fmaxf(0.f, fmaxf(xj.z - b1h.z, b1l.z - xj.z));
                push = gx * gx + gy * gy + gz * gz < rskip2;
            }
            const unsigned pb = __ballot_sync(0xffffffffu, push);
            if (push) {
                const int e = (q_head + q_len + __popc(pb & ((1u << lane) - 1u))) & (OG_JQ - 1);
                s_qx[wib][e] = xj;
                s_qi[wib][e] = make_int4(tj, c2 * OG_CELL + jj, (int)skip, img);
            }
            q_len += __popc(pb);
            __syncwarp();
            if (q_len >= 32) drain(32);
        }
        __syncwarp();  // the next chunk's survivors overwrite this chunk's
    }
    if (q_len > 0) drain(q_len);
    og_flush_icell<VIR, ENE>(A, c1, lane, frc, cell_acc);
}

// ---------------------------------------------------------------------------------------------
// j-list: the j-queue's two culls (cell2 box, then j atom, against cell1's box) done once per
// list build instead of every step.  k_jl_build keeps, per cell1, the (j atom, cell pair)
// entries whose j atom lies within cutoff + reach of cell1's bounding box; the step kernel
// k_pair_ljzd_jl streams them, 32 per round, one per lane.  reach = 2 skin + 1e-3 A: while no
// atom has moved farther than skin from the position the entries were built from (k_finish and
// k_put_state check this every step against xq_ref and set the stale counter otherwise), a
// dropped entry's pairs are farther apart than cutoff + 1e-3 A, so the step evaluates exactly
// the pairs the j-queue kernel evaluates.  The build runs at the first step of every list and
// after any stale mark; otherwise it returns at once.  Staleness is per system (jl_stale[s]):
// only the cells of a stale system are rebuilt, so a system's lists, and the order of its FP32
// i sums, are the ones it has alone in the engine.
//
// Entry: x = j slot | exclusion byte << 24 (slots below 2^24), y = cell-pair index.  Cell1's
// entries start at 8 * cp_head[c1] (at most 8 per cell pair), with their count in jl_count.
template <int NT>
__global__ void __launch_bounds__(NT)
k_jl_build(int *__restrict__ counters, const int *__restrict__ cell_sys, const SysDev *__restrict__ sys,
           const float4 *__restrict__ bbox, const float4 *__restrict__ xq, const int *__restrict__ cp_head,
           const float4 *__restrict__ cp_shift, const unsigned long long *__restrict__ cp_mask, long long pair_cap,
           float reach, int2 *__restrict__ jl, int *__restrict__ jl_count, float4 *__restrict__ xq_ref,
           const int *__restrict__ jl_stale) {
    if (counters[OG_CNT_JL_STALE] == 0) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) counters[OG_CNT_JL_BUILDS]++;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int jj = lane & 7, q = lane >> 3;
    const int n_cells = counters[OG_CNT_N_CELLS];
    __shared__ float4 s_sp[NT / 32][32];
    __shared__ uint2 s_m[NT / 32][32];
    __shared__ int s_k[NT / 32][32];
    const int c1 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (c1 >= n_cells) return;
    const int s1 = cell_sys[c1];
    if (!jl_stale[s1]) return;
    const SysDev &S = sys[s1];
    if (lane < OG_CELL) xq_ref[c1 * OG_CELL + lane] = xq[c1 * OG_CELL + lane];
    const float rb = sqrtf(S.cutoff2) + reach, rb2 = rb * rb;
    const float4 b1l = bbox[2 * c1], b1h = bbox[2 * c1 + 1];
    const long long k_beg = cp_head[c1];
    const long long k_end = min((long long)cp_head[c1 + 1], pair_cap);
    int2 *out = jl + 8 * k_beg;
    int count = 0;
    // each chunk's records are loaded while the previous chunk is processed
    float4 sp_next = make_float4(0.f, 0.f, 0.f, 0.f);
    unsigned long long m_next = ~0ull;
    if (k_beg + lane < k_end) {
        sp_next = cp_shift[k_beg + lane];
        m_next = cp_mask[k_beg + lane];
    }
    for (long long chunk = k_beg; chunk < k_end; chunk += 32) {
        const long long kk = chunk + lane;
        const float4 sp = sp_next;
        const unsigned long long m = m_next;
        if (kk + 32 < k_end) {
            sp_next = cp_shift[kk + 32];
            m_next = cp_mask[kk + 32];
        }
        bool keep = false;
        if (kk < k_end) {
            const int c2 = __float_as_int(sp.w);
            const float4 l2 = bbox[2 * c2], h2 = bbox[2 * c2 + 1];
            const float gx = fmaxf(0.f, fmaxf(l2.x + sp.x - b1h.x, b1l.x - (h2.x + sp.x)));
            const float gy = fmaxf(0.f, fmaxf(l2.y + sp.y - b1h.y, b1l.y - (h2.y + sp.y)));
            const float gz = fmaxf(0.f, fmaxf(l2.z + sp.z - b1h.z, b1l.z - (h2.z + sp.z)));
            keep = gx * gx + gy * gy + gz * gz < rb2;
        }
        const unsigned ballot = __ballot_sync(0xffffffffu, keep);
        const int n_keep = __popc(ballot);
        if (keep) {
            const int rank = __popc(ballot & ((1u << lane) - 1u));
            s_sp[wib][rank] = sp;
            s_m[wib][rank] = make_uint2((unsigned)m, (unsigned)(m >> 32));
            s_k[wib][rank] = (int)kk;
        }
        __syncwarp();
        // the survivors, four at a time (lane: survivor q, j atom jj); two such rounds per pass,
        // with both rounds' position loads issued before either is tested
        for (int r = 0; r < n_keep; r += 8) {
            float4 rsp[2], xj[2];
            unsigned skip[2];
            int rk[2];
            bool live[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int idx = r + 4 * h + q;
                const bool active = idx < n_keep;
                rsp[h] = make_float4(0.f, 0.f, 0.f, 0.f);
                unsigned long long rm = ~0ull;
                rk[h] = 0;
                if (active) {
                    rsp[h] = s_sp[wib][idx];
                    const uint2 mm = s_m[wib][idx];
                    rm = ((unsigned long long)mm.y << 32) | mm.x;
                    rk[h] = s_k[wib][idx];
                }
                skip[h] = active ? (unsigned)(rm >> (jj * OG_CELL)) & 0xffu : 0xffu;
                live[h] = active && skip[h] != 0xffu;
                xj[h] = live[h] ? xq[__float_as_int(rsp[h].w) * OG_CELL + jj] : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int c2 = __float_as_int(rsp[h].w);
                bool push = false;
                if (live[h]) {
                    const float x = xj[h].x + rsp[h].x, y = xj[h].y + rsp[h].y, z = xj[h].z + rsp[h].z;
                    const float gx = fmaxf(0.f, fmaxf(x - b1h.x, b1l.x - x));
                    const float gy = fmaxf(0.f, fmaxf(y - b1h.y, b1l.y - y));
                    const float gz = fmaxf(0.f, fmaxf(z - b1h.z, b1l.z - z));
                    push = gx * gx + gy * gy + gz * gz < rb2;
                }
                const unsigned pb = __ballot_sync(0xffffffffu, push);
                if (push)
                    out[count + __popc(pb & ((1u << lane) - 1u))] =
                        make_int2((int)((unsigned)(c2 * OG_CELL + jj) | (skip[h] << 24)), rk[h]);
                count += __popc(pb);
            }
        }
        __syncwarp();  // the next chunk's survivors overwrite this chunk's
    }
    if (lane == 0) jl_count[c1] = count;
}

// The step kernel over the j lists (see k_jl_build).  Each round, lane l takes entry r + l.
// The first block clears the stale marks: this launch follows the build that consumed them.
template <bool VIR, bool ENE, int MINB, int NT = 128, bool GEN = false>
__global__ void __launch_bounds__(NT, MINB)
k_pair_ljzd_jl(int *__restrict__ counters, const int *__restrict__ cell_sys, const SysDev *__restrict__ sys,
               const float4 *__restrict__ xq, const int *__restrict__ slot_type, const int *__restrict__ cp_head,
               const float4 *__restrict__ cp_shift, const int2 *__restrict__ cp_c2img, const int2 *__restrict__ jl,
               const int *__restrict__ jl_count, const float2 *__restrict__ lj, unsigned long long *__restrict__ frc,
               double *__restrict__ cell_acc, const EleDev *__restrict__ ele, const float2 *__restrict__ hps,
               int *__restrict__ jl_stale, int n_sys) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    if (blockIdx.x == 0) {
        if (threadIdx.x == 0) counters[OG_CNT_JL_STALE] = 0;
        for (int s = threadIdx.x; s < n_sys; s += NT) jl_stale[s] = 0;
    }
    const int n_cells = counters[OG_CNT_N_CELLS];
    if (warp >= n_cells) return;
    const int c1 = warp;
    const SysDev &S = sys[cell_sys[c1]];
    const EleDev &E = ele[GEN ? cell_sys[c1] : 0];
    __shared__ OgICell s_i[NT / 32];
    og_load_icell<GEN>(s_i[wib], c1, lane, xq, slot_type, S);
    const OgZdConst K = og_zd_const(S);
    OgIAcc<VIR> A;
    og_iacc_zero(A);
    const int2 *ent = jl + 8LL * cp_head[c1];
    const int n = jl_count[c1];
    // entries are loaded AHEAD rounds ahead and their gathers issued one round ahead; the
    // gathered values stay as loaded (position and cell-pair shift apart) until the round that
    // uses them, so neither load of the entry -> position chain is waited on in the round that
    // issues it.  Three rounds for the energy-free zero-dipole kernel; two where the energy or
    // generic terms leave no registers for the third (it spills there)
    constexpr int AHEAD = (ENE || GEN) ? 2 : 3;
    float4 g_xq = make_float4(0.f, 0.f, 0.f, 0.f), g_sp = make_float4(0.f, 0.f, 0.f, 0.f);
    int g_tj = 0, g_slot = 0, g_img = 0;
    unsigned g_skip = 0xffu;
    auto gather = [&](int2 e, bool ok) {
        if (ok) {
            g_slot = e.x & 0xffffff;
            g_skip = (unsigned)e.x >> 24;
            g_sp = cp_shift[e.y];
            g_xq = xq[g_slot];
            g_tj = slot_type[g_slot];
            if (VIR) g_img = cp_c2img[e.y].y;
        }
    };
    int2 e_ahead[AHEAD - 1];  // entries of rounds r + 1 .. r + AHEAD - 1
    if (lane < n) gather(ent[lane], true);
#pragma unroll
    for (int a = 0; a < AHEAD - 1; a++) {
        e_ahead[a] = make_int2(0, 0);
        if (32 * (a + 1) + lane < n) e_ahead[a] = ent[32 * (a + 1) + lane];
    }
    for (int r = 0; r < n; r += 32) {
        const bool active = r + lane < n;
        const float4 xj = make_float4(g_xq.x + g_sp.x, g_xq.y + g_sp.y, g_xq.z + g_sp.z, g_xq.w);
        const int tj = g_tj, slot = g_slot, img = g_img;
        const unsigned skip = active ? g_skip : 0xffu;
        const int2 e1 = e_ahead[0];
#pragma unroll
        for (int a = 0; a + 1 < AHEAD - 1; a++) e_ahead[a] = e_ahead[a + 1];
        if (r + 32 * AHEAD + lane < n) e_ahead[AHEAD - 2] = ent[r + 32 * AHEAD + lane];
        gather(e1, r + 32 + lane < n);
        og_eval_j<VIR, ENE, GEN>(A, active, xj, tj, skip, slot, img, s_i[wib], K, S, E, lj, hps, frc);
    }
    og_flush_icell<VIR, ENE>(A, c1, lane, frc, cell_acc);
}

// ---------------------------------------------------------------------------------------------
// FP64 evaluation of the cell-pair list (pair variant OG_PAIR_VARIANT_F64): the reference's pair
// terms (ForceField::calc_pairwise with ZeroMultipoleSum::calc_zero02pole_alpha0,
// ForceField.cpp:333-418, ZeroMultipoleSum.cpp:309-332) in double precision throughout, on the
// list's FP64 grid coordinates (MiniCell::crd), FP64 charges and an FP64 C6/C12 table, with the
// image shift of each cell pair formed from the float box length as PBC holds it.  A validation
// mode: it separates the FP32 arithmetic of the production kernels from everything else of a
// trajectory (list, integrator, constraints).  Zero-dipole alpha = 0 with plain LJ only.
// One warp per cell1: lane l takes i atom l & 7 and j atoms (l >> 3) and (l >> 3) + 4 of every
// cell pair; j work is reduced over the 8 lanes of a j atom, i work over the lanes of an i atom
// at the end, both added to the fixed-point accumulators.
template <bool VIR>
__global__ void __launch_bounds__(256)
k_pair_f64(const int *__restrict__ counters, const int *__restrict__ cell_sys, const SysDev *__restrict__ sys,
           const double *__restrict__ slot_crd, const int *__restrict__ slot_atom, const int *__restrict__ slot_type,
           const double *__restrict__ charge, const int *__restrict__ cp_head, const int2 *__restrict__ cp_c2img,
           const unsigned long long *__restrict__ cp_mask, const double2 *__restrict__ lj64, long long pair_cap,
           unsigned long long *__restrict__ frc, double *__restrict__ cell_acc) {
    const int c1 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int n_cells = counters[OG_CNT_N_CELLS];
    if (c1 >= n_cells) return;
    const SysDev &S = sys[cell_sys[c1]];
    const int a1 = lane & 7, h = lane >> 3;
    const int s1 = c1 * OG_CELL + a1;
    const double x1[3] = {slot_crd[3 * (size_t)s1], slot_crd[3 * (size_t)s1 + 1], slot_crd[3 * (size_t)s1 + 2]};
    const int at1 = slot_atom[s1];
    const double q1 = at1 >= 0 ? charge[at1] : 0.0;
    const int row1 = S.lj_base + slot_type[s1] * S.n_types;
    const double rc = S.cutoff, rc2 = rc * rc;
    const double fco = 1.0 / (rc * rc * rc), bco = 0.5 * fco, zco = 1.0 / rc + bco * rc * rc;
    const double Lb[3] = {(double)S.Lf[0], (double)S.Lf[1], (double)S.Lf[2]};
    double wi[3] = {0.0, 0.0, 0.0}, ev = 0.0, ee = 0.0, vir[VIR ? 9 : 1] = {};
    int n_act = 0;
    const long long k_beg = cp_head[c1], k_end = min((long long)cp_head[c1 + 1], pair_cap);
    for (long long k = k_beg; k < k_end; k++) {
        const int2 ci = cp_c2img[k];
        const unsigned long long m = cp_mask[k];
        const int img = ci.y;
        const double sh[3] = {(img & 1) ? -Lb[0] : ((img & 2) ? Lb[0] : 0.0),
                              (img & 4) ? -Lb[1] : ((img & 8) ? Lb[1] : 0.0),
                              (img & 16) ? -Lb[2] : ((img & 32) ? Lb[2] : 0.0)};
#pragma unroll
        for (int half = 0; half < 2; half++) {
            const int a2 = h + 4 * half;
            const int s2 = ci.x * OG_CELL + a2;
            double w[3] = {0.0, 0.0, 0.0};
            if (!((m >> (a2 * OG_CELL + a1)) & 1ull)) {
                double d[3];
                for (int q = 0; q < 3; q++) d[q] = x1[q] - (slot_crd[3 * (size_t)s2 + q] + sh[q]);
                const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
                if (r2 < rc2) {
                    const int at2 = slot_atom[s2];
                    const double cc = q1 * (at2 >= 0 ? charge[at2] : 0.0) * OG_CHARGE_COEFF;
                    const double2 c = lj64[row1 + slot_type[s2]];
                    const double r = sqrt(r2), ri = 1.0 / r, r2i = 1.0 / r2, r6i = r2i * r2i * r2i;
                    const double t6 = c.x * r6i, t12 = c.y * r6i * r6i;
                    ev += t12 - t6;
                    ee += cc * (ri - zco + bco * r2);
                    const double wc = r2i * (-12.0 * t12 + 6.0 * t6) - cc * (ri * r2i - fco);
                    for (int q = 0; q < 3; q++) w[q] = wc * d[q];
                    n_act++;
                }
            }
            for (int q = 0; q < 3; q++) wi[q] += w[q];
            // j work: the 8 lanes of this j atom
            double wj[3] = {w[0], w[1], w[2]};
            for (int q = 0; q < 3; q++)
                for (int o = 1; o < OG_CELL; o <<= 1) wj[q] += __shfl_xor_sync(0xffffffffu, wj[q], o);
            if (a1 == 0 && (wj[0] != 0.0 || wj[1] != 0.0 || wj[2] != 0.0)) {
                unsigned long long *fj = frc + 3 * (size_t)s2;
                for (int q = 0; q < 3; q++) atomicAdd(fj + q, (unsigned long long)og_to_fix(-wj[q]));
                if (VIR && img != 0)  // sum over pairs of d (x) f: the shift term takes -(work on j)
                    for (int a = 0; a < 3; a++)
                        for (int b = 0; b < 3; b++) vir[a * 3 + b] += sh[a] * wj[b];
            }
        }
    }
    for (int q = 0; q < 3; q++) {
        wi[q] += __shfl_xor_sync(0xffffffffu, wi[q], 8);
        wi[q] += __shfl_xor_sync(0xffffffffu, wi[q], 16);
    }
    if (lane < OG_CELL && (wi[0] != 0.0 || wi[1] != 0.0 || wi[2] != 0.0)) {
        unsigned long long *fa = frc + 3 * (size_t)s1;
        for (int q = 0; q < 3; q++) atomicAdd(fa + q, (unsigned long long)og_to_fix(wi[q]));
    }
    for (int o = 16; o > 0; o >>= 1) {
        ev += __shfl_xor_sync(0xffffffffu, ev, o);
        ee += __shfl_xor_sync(0xffffffffu, ee, o);
        n_act += __shfl_xor_sync(0xffffffffu, n_act, o);
        if (VIR)
            for (int k = 0; k < 9; k++) vir[k] += __shfl_xor_sync(0xffffffffu, vir[k], o);
    }
    if (lane == 0) {
        double *acc = cell_acc + (size_t)c1 * OG_CELL_ACC;
        acc[0] = ev;
        acc[1] = ee;
        if (VIR) {
            for (int k = 0; k < 9; k++) acc[2 + k] = vir[k];
            acc[11] = (double)n_act;
        }
    }
}

#define OG_PAIR_ARGS_DECL                                                                                   \
    const int *, const int *, const SysDev *, const float4 *, const float4 *, const int *, const int *,      \
        const float4 *, const int2 *, const unsigned long long *, const float2 *, unsigned long long *, double *, \
        long long
template __global__ void k_pair_ljzd_jm<true, 2>(OG_PAIR_ARGS_DECL);
template __global__ void k_pair_ljzd_jm<false, 2>(OG_PAIR_ARGS_DECL);
template __global__ void k_pair_ljzd_jm<false, 3>(OG_PAIR_ARGS_DECL);
template __global__ void k_pair_ljzd_jm2<true, true, 2>(OG_PAIR_ARGS_DECL);
template __global__ void k_pair_ljzd_jm2<false, true, 2>(OG_PAIR_ARGS_DECL);
template __global__ void k_pair_ljzd_jm2<false, true, 3>(OG_PAIR_ARGS_DECL);
template __global__ void k_pair_ljzd_jm2<false, false, 2>(OG_PAIR_ARGS_DECL);
template __global__ void k_pair_ljzd_jm2<false, false, 3>(OG_PAIR_ARGS_DECL);
#define OG_JQ_ARGS_DECL OG_PAIR_ARGS_DECL, const EleDev *, const float2 *
template __global__ void k_pair_ljzd_jq<true, true, 2, 256, false>(OG_JQ_ARGS_DECL);
template __global__ void k_pair_ljzd_jq<false, true, 2, 256, false>(OG_JQ_ARGS_DECL);
template __global__ void k_pair_ljzd_jq<false, true, 3, 256, false>(OG_JQ_ARGS_DECL);
template __global__ void k_pair_ljzd_jq<false, false, 2, 256, false>(OG_JQ_ARGS_DECL);
template __global__ void k_pair_ljzd_jq<false, false, 3, 256, false>(OG_JQ_ARGS_DECL);
template __global__ void k_pair_ljzd_jq<false, true, 5, 128, false>(OG_JQ_ARGS_DECL);
template __global__ void k_pair_ljzd_jq<false, false, 5, 128, false>(OG_JQ_ARGS_DECL);
template __global__ void k_pair_ljzd_jq<true, true, 2, 256, true>(OG_JQ_ARGS_DECL);
template __global__ void k_pair_ljzd_jq<false, true, 5, 128, true>(OG_JQ_ARGS_DECL);
template __global__ void k_pair_ljzd_jq<false, false, 5, 128, true>(OG_JQ_ARGS_DECL);
#define OG_JL_ARGS_DECL                                                                                    \
    int *, const int *, const SysDev *, const float4 *, const int *, const int *, const float4 *, const int2 *, \
        const int2 *, const int *, const float2 *, unsigned long long *, double *, const EleDev *, const float2 *, \
        int *, int
template __global__ void k_pair_ljzd_jl<true, true, 2, 128, false>(OG_JL_ARGS_DECL);
template __global__ void k_pair_ljzd_jl<false, true, 5, 128, false>(OG_JL_ARGS_DECL);
template __global__ void k_pair_ljzd_jl<false, false, 5, 128, false>(OG_JL_ARGS_DECL);
template __global__ void k_pair_ljzd_jl<true, true, 2, 128, true>(OG_JL_ARGS_DECL);
template __global__ void k_pair_ljzd_jl<false, true, 5, 128, true>(OG_JL_ARGS_DECL);
template __global__ void k_pair_ljzd_jl<false, false, 5, 128, true>(OG_JL_ARGS_DECL);
#define OG_F64_ARGS_DECL                                                                                   \
    const int *, const int *, const SysDev *, const double *, const int *, const int *, const double *,      \
        const int *, const int2 *, const unsigned long long *, const double2 *, long long, unsigned long long *, \
        double *
template __global__ void k_pair_f64<true>(OG_F64_ARGS_DECL);
template __global__ void k_pair_f64<false>(OG_F64_ARGS_DECL);
template __global__ void k_jl_build<256>(int *, const int *, const SysDev *, const float4 *, const float4 *,
                                         const int *, const float4 *, const unsigned long long *, long long, float,
                                         int2 *, int *, float4 *, const int *);

template __global__ void k_pair_ljzd<true, 2>(const int *, const int *, const SysDev *, const float4 *,
                                                const float4 *, const int *, const int *, const float4 *,
                                                const int2 *, const unsigned long long *, const float2 *,
                                                unsigned long long *, double *, long long);
template __global__ void k_pair_ljzd<true, 3>(const int *, const int *, const SysDev *, const float4 *,
                                                const float4 *, const int *, const int *, const float4 *,
                                                const int2 *, const unsigned long long *, const float2 *,
                                                unsigned long long *, double *, long long);
template __global__ void k_pair_ljzd<true, 4>(const int *, const int *, const SysDev *, const float4 *,
                                                const float4 *, const int *, const int *, const float4 *,
                                                const int2 *, const unsigned long long *, const float2 *,
                                                unsigned long long *, double *, long long);
template __global__ void k_pair_ljzd<false, 2>(const int *, const int *, const SysDev *, const float4 *,
                                                const float4 *, const int *, const int *, const float4 *,
                                                const int2 *, const unsigned long long *, const float2 *,
                                                unsigned long long *, double *, long long);
template __global__ void k_pair_ljzd<false, 3>(const int *, const int *, const SysDev *, const float4 *,
                                                const float4 *, const int *, const int *, const float4 *,
                                                const int2 *, const unsigned long long *, const float2 *,
                                                unsigned long long *, double *, long long);
template __global__ void k_pair_ljzd<false, 4>(const int *, const int *, const SysDev *, const float4 *,
                                                const float4 *, const int *, const int *, const float4 *,
                                                const int2 *, const unsigned long long *, const float2 *,
                                                unsigned long long *, double *, long long);

}  // namespace og
