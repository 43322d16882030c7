// og_integrate.cu -- everything of the per-step path except the cell list and the pair kernel:
// excluded-pair ZD correction, bonds/angles, fixed-point -> FP64 work, V-McMD force scaling,
// the leapfrog-presto update, COM cancel, SHAKE pair/trio, velocity-scaling thermostat (with
// and without constraints), grid move, PBC wrap, kinetic energy and the fixed-order
// per-system reductions.  One thread per atom / constraint / term; every kernel covers all
// systems of the batch.  All integrator arithmetic is FP64 (the reference's `real`).
#include "og_internal.cuh"

namespace og {

// ------------------------------------------------------------- helpers

// Minimum image of PBC::diff_crd_minim_image, double overload (PBC.cpp:70-84): the reference
// truncates d * (1 / (L/2)) to int twice, with float box lengths.  Where float(2/L) * L rounds
// above 2 (a 97.26 A box: by 8.8e-8), a difference within L * (L*lhi/2 - 1) of +-L (4.3e-6 A
// there) cycles +L -> -L through the two truncations and comes back as +-L instead of ~0: two
// atoms of one molecule on opposite faces with x offsets that agree to a few microangstroms
// get a bond, angle or constraint vector one box long (the reference's SHAKE then diverges and
// throws the molecule across the box).  The third pass fires only on that result (|d| > 3L/4;
// every other result of the two passes is within L/2 of 0), so all others are the reference's
// bit for bit.
__device__ __forceinline__ double minim(double d, float L, float lhi) {
    d = d - (double)(L * (float)(int)(d * (double)lhi));
    d = d - (double)(L * (float)(int)(d * (double)lhi));
    if (fabs(d) > 0.75 * (double)L) d = d > 0.0 ? d - (double)L : d + (double)L;
    return d;
}

__device__ __forceinline__ void add_fix(unsigned long long *f, double wx, double wy, double wz) {
    atomicAdd(f + 0, (unsigned long long)og_to_fix(wx));
    atomicAdd(f + 1, (unsigned long long)og_to_fix(wy));
    atomicAdd(f + 2, (unsigned long long)og_to_fix(wz));
}

// ------------------------------------------------------------- forces

// Excluded-pair ("excess") zero-dipole term, E = cc bcoeff r^2, dE/dx = cc fcoeff d
// (ForceField.cpp:420-437, ZeroMultipoleSum.cpp:191-202, SubBox.cpp:1347-1367), in FP64.
// The excluded-pair term of models other than zero-dipole alpha = 0 in FP64
// (ZeroMultipoleSum.cpp:204-307; Debye-Hueckel has none, calc_null), with the reference's forms:
// the zero-dipole alpha > 0 energy takes -erf(alpha r) r, the octupole energies r^4 r, the
// hexadecapole alpha = 0 gradient zh66 r^2 and -1/r^3, the hexadecapole alpha > 0 energy stops at r^4.
__device__ void og_ele_excess(const EleDev &E, double r, double r2, double cc, double &e, double &g) {
    e = g = 0.0;
    if (E.mode == OG_ELE_DH) return;
    const double ri = 1.0 / r, r2i = ri * ri, r3i = r2i * ri, r4 = r2 * r2, r6 = r4 * r2, r8 = r4 * r4;
    double erc = 1.0, erfn = 0.0, ex = 0.0;
    if (!E.alpha0) {
        const double t = E.d_alpha * r;
        erc = erfc(t);
        erfn = 1.0 - erc;
        ex = E.d_piewald * exp(-t * t) * r2i;
    }
    switch (E.mode) {
        case OG_ELE_ZD:
            if (E.alpha0) {
                e = cc * E.d_bcoeff * r2;
                g = cc * E.d_fcoeff;
            } else {
                e = cc * (-erfn * r + E.d_bcoeff * r2);
                g = -cc * (erc * r3i + ex - E.d_fcoeff - r3i);
            }
            break;
        case OG_ELE_ZQ:
            e = cc * (-erfn * ri - E.d_zq2 * r2 - E.d_zq4 * r4);
            g = -cc * (E.alpha0 ? (E.d_zq22 + E.d_zq44 * r2) : (erc * r3i + ex + E.d_zq22 + E.d_zq44 * r2 - r3i));
            break;
        case OG_ELE_ZO:
            e = cc * (-erfn * ri - E.d_zo2 * r2 - E.d_zo4 * r4 - E.d_zo6 * r4 * r);
            g = -cc * (E.alpha0 ? (E.d_zo22 + E.d_zo44 * r2 + E.d_zo66 * r4)
                                : (erc * r3i + ex + E.d_zo22 + E.d_zo44 * r2 + E.d_zo66 * r4 - r3i));
            break;
        default:
            if (E.alpha0) {
                e = cc * (-E.d_zh2 * r2 - E.d_zh4 * r4 - E.d_zh6 * r6 - E.d_zh8 * r8);
                g = -cc * (E.d_zh22 + E.d_zh44 * r2 + E.d_zh66 * r2 + E.d_zh88 * r6 - r3i);
            } else {
                e = cc * (-erfn * ri - E.d_zh2 * r2 - E.d_zh4 * r4);
                g = -cc * (erc * r3i + ex + E.d_zh22 + E.d_zh44 * r2 + E.d_zh66 * r4 + E.d_zh88 * r6 - r3i);
            }
    }
}

__global__ void k_excess(int n_pairs, const int2 *__restrict__ pairs, const int *__restrict__ pair_sys,
                         const SysDev *__restrict__ sys, const EleDev *__restrict__ ele,
                         const double *__restrict__ crd, const double *__restrict__ charge,
                         const int *__restrict__ atom_slot, unsigned long long *__restrict__ frc,
                         double *__restrict__ e_out, double *__restrict__ vir_out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_pairs) return;
    const int s = pair_sys[k];
    const SysDev &S = sys[s];
    const int i = pairs[k].x, j = pairs[k].y;
    double d[3];
    for (int q = 0; q < 3; q++) d[q] = minim(crd[3 * i + q] - crd[3 * j + q], S.Lf[q], S.L_half_inv_f[q]);
    const double cc = charge[i] * charge[j] * OG_CHARGE_COEFF;
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    double gc;
    if (!ele[s].generic) {
        const double fco = 1.0 / (S.cutoff * S.cutoff * S.cutoff);
        e_out[k] = cc * 0.5 * fco * r2;
        gc = cc * fco;
    } else {
        double e;
        og_ele_excess(ele[s], sqrt(r2), r2, cc, e, gc);
        e_out[k] = e;
    }
    add_fix(frc + 3 * (size_t)atom_slot[i], gc * d[0], gc * d[1], gc * d[2]);
    add_fix(frc + 3 * (size_t)atom_slot[j], -gc * d[0], -gc * d[1], -gc * d[2]);
    if (vir_out)
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) vir_out[9 * (size_t)k + a * 3 + b] = -d[a] * gc * d[b];
}

// Harmonic bonds E = k (r - r0)^2 (ForceField.cpp:108-128).
__global__ void k_bonds(int n, const int2 *__restrict__ b, const double2 *__restrict__ kr,
                        const int *__restrict__ bsys, const SysDev *__restrict__ sys,
                        const double *__restrict__ crd, const int *__restrict__ atom_slot,
                        unsigned long long *__restrict__ frc, double *__restrict__ e_out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const SysDev &S = sys[bsys[k]];
    const int i = b[k].x, j = b[k].y;
    double d[3];
    for (int q = 0; q < 3; q++) d[q] = minim(crd[3 * i + q] - crd[3 * j + q], S.Lf[q], S.L_half_inv_f[q]);
    const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    const double dif = r - kr[k].y, coef = kr[k].x * dif;
    e_out[k] = coef * dif;
    const double gc = 2.0 * coef / r;
    add_fix(frc + 3 * (size_t)atom_slot[i], d[0] * gc, d[1] * gc, d[2] * gc);
    add_fix(frc + 3 * (size_t)atom_slot[j], -d[0] * gc, -d[1] * gc, -d[2] * gc);
}

// Harmonic angles E = k (theta - theta0)^2 (ForceField.cpp:130-177).
__global__ void k_angles(int n, const int4 *__restrict__ a, const double2 *__restrict__ kt,
                         const SysDev *__restrict__ sys, const double *__restrict__ crd,
                         const int *__restrict__ atom_slot, unsigned long long *__restrict__ frc,
                         double *__restrict__ e_out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const SysDev &S = sys[a[k].w];
    const int i = a[k].x, j = a[k].y, l = a[k].z;
    double d12[3], d32[3];
    for (int q = 0; q < 3; q++) {
        d12[q] = minim(crd[3 * i + q] - crd[3 * j + q], S.Lf[q], S.L_half_inv_f[q]);
        d32[q] = minim(crd[3 * l + q] - crd[3 * j + q], S.Lf[q], S.L_half_inv_f[q]);
    }
    const double r12_2 = d12[0] * d12[0] + d12[1] * d12[1] + d12[2] * d12[2];
    const double r32_2 = d32[0] * d32[0] + d32[1] * d32[1] + d32[2] * d32[2];
    const double rri = 1.0 / sqrt(r12_2 * r32_2);
    double cost = (d12[0] * d32[0] + d12[1] * d32[1] + d12[2] * d32[2]) * rri;
    cost = fmax(fmin(cost, 1.0), -1.0);
    const double th = acos(cost);
    const double dif = th - kt[k].y, coef = kt[k].x * dif;
    e_out[k] = coef * dif;
    const double r12i = 1.0 / r12_2, r32i = 1.0 / r32_2;
    const double st = fmax(1e-10, sin(th));
    const double gc = -(2.0 * coef) / st;
    double w1[3], w2[3];
    for (int q = 0; q < 3; q++) {
        w1[q] = gc * (d32[q] * rri - d12[q] * cost * r12i);
        w2[q] = gc * (d12[q] * rri - d32[q] * cost * r32i);
    }
    add_fix(frc + 3 * (size_t)atom_slot[i], w1[0], w1[1], w1[2]);
    add_fix(frc + 3 * (size_t)atom_slot[j], -w1[0] - w2[0], -w1[1] - w2[1], -w1[2] - w2[2]);
    add_fix(frc + 3 * (size_t)atom_slot[l], w2[0], w2[1], w2[2]);
}

__device__ __forceinline__ void cross3(const double a[3], const double b[3], double c[3]) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

// Dihedral terms, E = ene (1 + cos(n phi - phase)) / overlaps, in FP64 (ForceField::calc_torsion,
// ForceField.cpp:179-300, applied as SubBox::calc_energy_torsions / calc_energy_impros,
// SubBox.cpp:1273-1320); one launch for torsions and one for impropers.  prm[k] = (ene, phase,
// overlaps, symmetry).  The reference's PI (CelesteObject.cpp:27) and its table of 2k for even
// multiplicities (ForceField.cpp:7-17) are part of the arithmetic.
__global__ void k_dihedrals(int n, const int4 *__restrict__ q4, const double4 *__restrict__ prm,
                            const int *__restrict__ dsys, const SysDev *__restrict__ sys,
                            const double *__restrict__ crd, const int *__restrict__ atom_slot,
                            unsigned long long *__restrict__ frc, double *__restrict__ e_out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const SysDev &S = sys[dsys[k]];
    const int a1 = q4[k].x, a2 = q4[k].y, a3 = q4[k].z, a4 = q4[k].w;
    const double4 P = prm[k];
    double w1[3] = {0, 0, 0}, w2[3] = {0, 0, 0}, w3[3] = {0, 0, 0}, e = 0.0;
    if (P.x > 1e-10) {
        double d21[3], d32[3], d43[3], p12[3], p23[3], p123[3];
        for (int q = 0; q < 3; q++) {
            d21[q] = minim(crd[3 * a2 + q] - crd[3 * a1 + q], S.Lf[q], S.L_half_inv_f[q]);
            d32[q] = minim(crd[3 * a3 + q] - crd[3 * a2 + q], S.Lf[q], S.L_half_inv_f[q]);
            d43[q] = minim(crd[3 * a4 + q] - crd[3 * a3 + q], S.Lf[q], S.L_half_inv_f[q]);
        }
        cross3(d21, d32, p12);
        cross3(d32, d43, p23);
        const double p12_2 = p12[0] * p12[0] + p12[1] * p12[1] + p12[2] * p12[2];
        const double p23_2 = p23[0] * p23[0] + p23[1] * p23[1] + p23[2] * p23[2];
        const double p12p23 = sqrt(p12_2 * p23_2);
        if (p12p23 > 0.0) {
            const double inv = 1.0 / p12p23;
            const double s1223 = p12[0] * p23[0] + p12[1] * p23[1] + p12[2] * p23[2];
            const double cosp = fmax(-1.0, fmin(1.0, s1223 * inv));
            cross3(p12, p23, p123);
            double phi = acos(cosp);
            if (d32[0] * p123[0] + d32[1] * p123[1] + d32[2] * p123[2] < 0.0) phi = 2.0 * 3.14159265 - phi;
            const double sym = P.w, div = 1.0 / P.z;
            e = P.x * (1.0 + cos(sym * phi - P.y)) * div;
            const int nrot = (int)sym;
            const double gm = (nrot >= 0 && nrot <= 10 && nrot % 2 == 0) ? (double)nrot : 0.0;
            const double sinp = sin(phi);
            const double sf = sin(P.y), cf = cos(P.y), sr = sin(sym * phi), cr = cos(sym * phi);
            const double dflim = cf * (sym - gm + gm * cosp);
            const double df0 = cf * sr - sf * cr;
            const double df1 = (1e-10 <= fabs(sinp)) ? df0 / sinp : dflim;
            const double wc = sym * P.x * div * df1 * inv;
            const double r12 = 1.0 / p12_2 * s1223, r23 = 1.0 / p23_2 * s1223;
            double a[3], b[3], c[3], dd[3];
            cross3(p23, d32, a);
            cross3(p12, d32, b);
            for (int i = 0; i < 3; i++) w1[i] = wc * (a[i] - r12 * b[i]);
            const double d2132[3] = {d21[0] + d32[0], d21[1] + d32[1], d21[2] + d32[2]};
            cross3(d2132, p23, a);
            cross3(d2132, p12, b);
            cross3(p12, d43, c);
            cross3(p23, d43, dd);
            for (int i = 0; i < 3; i++) w2[i] = wc * (a[i] + c[i] - r12 * b[i] - r23 * dd[i]);
            cross3(p12, d32, a);
            cross3(p23, d32, b);
            for (int i = 0; i < 3; i++) w3[i] = wc * (a[i] - r23 * b[i]);
        }
    }
    e_out[k] = e;
    add_fix(frc + 3 * (size_t)atom_slot[a1], w1[0], w1[1], w1[2]);
    add_fix(frc + 3 * (size_t)atom_slot[a2], w2[0], w2[1], w2[2]);
    add_fix(frc + 3 * (size_t)atom_slot[a3], -(w1[0] + w2[0] + w3[0]), -(w1[1] + w2[1] + w3[1]),
            -(w1[2] + w2[2] + w3[2]));
    add_fix(frc + 3 * (size_t)atom_slot[a4], w3[0], w3[1], w3[2]);
}

// 1-4 pairs (ForceField::calc_14pair, ForceField.cpp:302-331, via SubBox::calc_energy_14nb,
// SubBox.cpp:1321-1345): scaled LJ and Coulomb without cutoff, FP64 on the reference's float
// charges and LJ terms.  e_out[2k] = vdw, e_out[2k+1] = ele.
__global__ void k_nb14(int n, const int2 *__restrict__ pr, const int2 *__restrict__ ty,
                       const double2 *__restrict__ coef, const int *__restrict__ psys,
                       const SysDev *__restrict__ sys, const double *__restrict__ crd,
                       const float *__restrict__ charge_f, const float2 *__restrict__ lj,
                       const int *__restrict__ atom_slot, unsigned long long *__restrict__ frc,
                       double *__restrict__ e_out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const SysDev &S = sys[psys[k]];
    const int i = pr[k].x, j = pr[k].y;
    double d[3];
    for (int q = 0; q < 3; q++) d[q] = minim(crd[3 * i + q] - crd[3 * j + q], S.Lf[q], S.L_half_inv_f[q]);
    const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const double r2i = 1.0 / r2, ri = sqrt(r2i);
    const double r6i = r2i * r2i * r2i, r12i = r6i * r6i;
    const float2 p = lj[S.lj_base + ty[k].x * S.n_types + ty[k].y];
    const double t6 = (double)p.x * r6i, t12 = (double)p.y * r12i;
    const double cv = coef[k].x, ce = coef[k].y;
    e_out[2 * k] = (-t6 + t12) * cv;
    const double cw = r2i * cv * (-12.0 * t12 + 6.0 * t6);
    const double cc = (double)charge_f[i] * (double)charge_f[j] * OG_CHARGE_COEFF * ce;
    e_out[2 * k + 1] = cc * ri;
    const double cel = -cc * r2i * ri;
    const double w[3] = {cw * d[0] + cel * d[0], cw * d[1] + cel * d[1], cw * d[2] + cel * d[2]};
    add_fix(frc + 3 * (size_t)atom_slot[i], w[0], w[1], w[2]);
    add_fix(frc + 3 * (size_t)atom_slot[j], -w[0], -w[1], -w[2]);
}

// Per-atom x (x) F of the pair forces alone (virial, single-sum form); positions are the
// cell-relative coordinates the pair kernel used plus their cell origin.
__global__ void k_atom_virial(int n_atoms, const int *__restrict__ atom_slot,
                              const unsigned long long *__restrict__ frc, const float4 *__restrict__ xq,
                              const double *__restrict__ cell_origin, double *__restrict__ vir_out) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_atoms) return;
    const int s = atom_slot[a], c = s >> 3;
    const float4 p = xq[s];
    const double x[3] = {cell_origin[3 * c] + p.x, cell_origin[3 * c + 1] + p.y, cell_origin[3 * c + 2] + p.z};
    double F[3];
    for (int q = 0; q < 3; q++) F[q] = -(double)(long long)frc[3 * (size_t)s + q] * OG_FIX_INV;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) vir_out[9 * (size_t)a + i * 3 + j] = x[i] * F[j];
}

// Fixed-point accumulators -> FP64 work in atom order, clearing the accumulators.  One thread
// per slot: it reads its slot's three sums and clears them (coalesced), and writes the atom's
// work in original order (one 24-byte scatter).
__global__ void k_collect_slots(const int *__restrict__ counters, int slots_cap, const int *__restrict__ slot_atom,
                                unsigned long long *__restrict__ frc, double *__restrict__ work) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= slots_cap || s >= counters[OG_CNT_N_CELLS] * OG_CELL) return;
    const int a = slot_atom[s];
    unsigned long long *f = frc + 3 * (size_t)s;
    const long long f0 = (long long)f[0], f1 = (long long)f[1], f2 = (long long)f[2];
    f[0] = 0ull;
    f[1] = 0ull;
    f[2] = 0ull;
    if (a < 0) return;
    work[3 * (size_t)a + 0] = (double)f0 * OG_FIX_INV;
    work[3 * (size_t)a + 1] = (double)f1 * OG_FIX_INV;
    work[3 * (size_t)a + 2] = (double)f2 * OG_FIX_INV;
}

// ------------------------------------------------------------- reductions

// Block-wide sum of NV doubles per thread in a fixed order (deterministic).
template <int NV>
__device__ void block_sum(double (&v)[NV], double *sh) {
    const int t = threadIdx.x;
    for (int q = 0; q < NV; q++) sh[q * blockDim.x + t] = v[q];
    __syncthreads();
    for (int off = blockDim.x >> 1; off > 0; off >>= 1) {
        if (t < off)
            for (int q = 0; q < NV; q++) sh[q * blockDim.x + t] += sh[q * blockDim.x + t + off];
        __syncthreads();
    }
    for (int q = 0; q < NV; q++) v[q] = sh[q * blockDim.x];
    __syncthreads();
}

// Two-level fixed-order reductions.  Level 1: block (chunk, segment) sums NV fields of the
// items [base[s] + chunk*OG_RCHUNK, ...) of segment s; level 2: one block per segment sums its
// chunks in order.  Chunks are relative to the segment start, so a system's sums do not depend
// on what else is in the batch.
#define OG_RCHUNK 4096
template <int NV>
__global__ void k_part(const double *__restrict__ v, int stride, int field0, const int *__restrict__ base,
                       int max_chunks, double *__restrict__ part) {
    __shared__ double sh[NV * 256];
    const int s = blockIdx.y, ch = blockIdx.x;
    const long long b = (long long)base[s] + (long long)ch * OG_RCHUNK;
    const long long e = min((long long)base[s + 1], b + OG_RCHUNK);
    double acc[NV];
    for (int q = 0; q < NV; q++) acc[q] = 0.0;
    for (long long i = b + threadIdx.x; i < e; i += blockDim.x)
        for (int q = 0; q < NV; q++) acc[q] += v[i * stride + field0 + q];
    block_sum<NV>(acc, sh);
    if (threadIdx.x == 0)
        for (int q = 0; q < NV; q++) part[((size_t)s * max_chunks + ch) * NV + q] = acc[q];
}

// Level 1 for COM groups: momentum sum m v over a group's atom list.
__global__ void k_part_momentum(const int *__restrict__ grp_start, const int *__restrict__ grp_atoms,
                                const float *__restrict__ mass, const double *__restrict__ v,
                                const int *__restrict__ grp_sys, const int *__restrict__ sys_active, int max_chunks,
                                double *__restrict__ part) {
    __shared__ double sh[3 * 256];
    const int g = blockIdx.y, ch = blockIdx.x;
    const int b = grp_start[g] + ch * OG_RCHUNK;
    const int e = min(grp_start[g + 1], b + OG_RCHUNK);
    double m[3] = {0, 0, 0};
    if (sys_active == nullptr || sys_active[grp_sys[g]])
        for (int k = b + threadIdx.x; k < e; k += blockDim.x) {
            const int a = grp_atoms[k];
            for (int q = 0; q < 3; q++) m[q] += v[3 * a + q] * (double)mass[a];
        }
    block_sum<3>(m, sh);
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; q++) part[((size_t)g * max_chunks + ch) * 3 + q] = m[q];
}

// Level 2: out[s*out_stride + out_off + q] = (sum over chunks of part) * (scale ? scale[s] : 1).
template <int NV>
__global__ void k_part_final(const double *__restrict__ part, int max_chunks, double *__restrict__ out,
                             int out_stride, int out_off, const float *__restrict__ scale, int accumulate) {
    __shared__ double sh[NV * 256];
    const int s = blockIdx.x;
    double acc[NV];
    for (int q = 0; q < NV; q++) acc[q] = 0.0;
    for (int c = threadIdx.x; c < max_chunks; c += blockDim.x)
        for (int q = 0; q < NV; q++) acc[q] += part[((size_t)s * max_chunks + c) * NV + q];
    block_sum<NV>(acc, sh);
    if (threadIdx.x == 0)
        for (int q = 0; q < NV; q++) {
            const double r = acc[q] * (scale ? (double)scale[s] : 1.0);
            double &o = out[(size_t)s * out_stride + out_off + q];
            o = accumulate ? o + r : r;
        }
}

template __global__ void k_part<1>(const double *, int, int, const int *, int, double *);
template __global__ void k_part<2>(const double *, int, int, const int *, int, double *);
template __global__ void k_part<9>(const double *, int, int, const int *, int, double *);
template __global__ void k_part<10>(const double *, int, int, const int *, int, double *);
template __global__ void k_part_final<1>(const double *, int, double *, int, int, const float *, int);
template __global__ void k_part_final<2>(const double *, int, double *, int, int, const float *, int);
template __global__ void k_part_final<3>(const double *, int, double *, int, int, const float *, int);
template __global__ void k_part_final<9>(const double *, int, double *, int, int, const float *, int);
template __global__ void k_part_final<10>(const double *, int, double *, int, int, const float *, int);

// ------------------------------------------------------------------ V-McMD
// std::mt19937: the Mersenne Twister of Matsumoto & Nishimura (ACM TOMACS 8, 1998) with the
// parameters the C++ standard gives mt19937 ([rand.predef]: n 624, m 397, r 31, a 0x9908b0df,
// tempering u 11, s 7 b 0x9d2c5680, t 15 c 0xefc60000, l 18).  The reference draws
// generator() / double(generator.max()) (random::Random::operator(), Random.cpp:25-28).
// State: 624 words and the next position in word 624.  One warp advances a generator; the
// twist runs in two data-parallel ranges: words 0..226 read only old words, words 227..622 read
// the word 227 places back, already new, and word 623 reads new words 396 and 0.
__device__ __forceinline__ unsigned og_mt_mix(unsigned a, unsigned b, unsigned c) {
    const unsigned y = (a & 0x80000000u) | (b & 0x7fffffffu);
    return c ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
}

__device__ void og_mt_twist_warp(unsigned *st, int lane) {
    for (int b = 0; b < 227; b += 32) {
        const int i = b + lane;
        unsigned v = 0;
        if (i < 227) v = og_mt_mix(st[i], st[i + 1], st[i + 397]);
        __syncwarp();
        if (i < 227) st[i] = v;
        __syncwarp();
    }
    // a 32-word block [b, b+32) with b >= 227 reads words i-227 < b: all rewritten before it
    for (int b = 227; b < 623; b += 32) {
        const int i = b + lane;
        unsigned v = 0;
        if (i < 623) v = og_mt_mix(st[i], st[i + 1], st[i - 227]);
        __syncwarp();
        if (i < 623) st[i] = v;
        __syncwarp();
    }
    if (lane == 0) st[623] = og_mt_mix(st[623], st[0], st[396]);
    __syncwarp();
}

// Next tempered word; every lane of the warp calls it with the same position.
__device__ unsigned og_mt_next(unsigned *st, int &pos, int lane) {
    if (pos >= 624) {
        og_mt_twist_warp(st, lane);
        pos = 0;
    }
    unsigned y = st[pos++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

__device__ __forceinline__ bool og_vs_in_range(const VsDev &v, double lambda) {
    return lambda >= v.lo && lambda <= v.hi;  // VirtualState::is_in_range, Extend.cpp:53-55
}

// ExtendedVMcMD::trial_transition (Extend.cpp:160-177): a draw is made only when the neighbour
// state exists and holds lambda; the move is taken when the draw exceeds 1 - probability.
__device__ int og_vs_trial(const VsDev *V, int n_vs, int src, int rel, double lambda, unsigned *st, int &pos,
                           int lane) {
    if (!og_vs_in_range(V[src], lambda)) return src;
    if (src == 0 && rel == -1) return src;
    if (src == n_vs - 1 && rel == 1) return src;
    if (og_vs_in_range(V[src + rel], lambda)) {
        const double rnd = (double)og_mt_next(st, pos, lane) / 4294967295.0;
        const double prob = rel == 1 ? V[src].p_up : V[src].p_down;
        if (rnd > (1.0 - prob)) return src + rel;
    }
    return src;
}

// V-McMD per step, one warp per system (ExtendedVMcMD::apply_bias, Extend.cpp:126-143): the
// step's potential is lambda (MmSystem::set_potential_e); at a transition step the state moves
// (set_current_vstate, Extend.cpp:144-158) and is logged, every lambda-log step lambda is logged,
// and the force factor is const_k * the state's polynomial at lambda clamped to the state's range
// (scale_force, Extend.cpp:178-203).  advance = 0 (a force evaluation outside a step) leaves the
// state, generator and logs alone.
__global__ void k_vmcmd(int n_sys, const SysDev *__restrict__ sys, const VsDev *__restrict__ vstates,
                        const double *__restrict__ sys_acc, const long long *__restrict__ step, int advance,
                        int *__restrict__ vs_cur, unsigned *__restrict__ mt, int *__restrict__ vs_log,
                        double *__restrict__ lambda_log, int log_cap, double *__restrict__ mcmd_factor) {
    const int s = blockIdx.x, lane = threadIdx.x;
    if (s >= n_sys) return;
    const SysDev &S = sys[s];
    if (S.n_vs == 0) {
        if (lane == 0) mcmd_factor[s] = 1.0;
        return;
    }
    const double *acc = sys_acc + OG_ACC_SIZE * s;
    // MmSystem::set_potential_e's order (MmSystem.cpp:738-742)
    const double lambda = acc[OG_ACC_BOND] + acc[OG_ACC_ANGLE] + acc[OG_ACC_TORSION] + acc[OG_ACC_IMPRO] +
                          acc[OG_ACC_VDW14] + acc[OG_ACC_ELE14] + acc[OG_ACC_VDW] +
                          (acc[OG_ACC_ELE] + acc[OG_ACC_EXCESS] + S.self_energy);
    const VsDev *V = vstates + S.vs_base;
    int cur = vs_cur[s];
    if (advance && S.vm_slot >= 0) {
        const long long g = *step + S.first_step;
        const size_t ring = (size_t)S.vm_slot * log_cap;
        if (g > 0 && g % S.vs_trans_intvl == 0) {
            unsigned *st = mt + (size_t)OG_MT_WORDS * S.vm_slot;
            int pos = (int)st[624];
            int dest = og_vs_trial(V, S.n_vs, cur, 1, lambda, st, pos, lane);
            if (dest == cur) dest = og_vs_trial(V, S.n_vs, cur, -1, lambda, st, pos, lane);
            cur = dest;
            __syncwarp();
            if (lane == 0) {
                st[624] = (unsigned)pos;
                vs_cur[s] = cur;
                vs_log[ring + (size_t)((g / S.vs_trans_intvl - 1) % log_cap)] = cur;
            }
        }
        if (lane == 0 && g > 0 && S.vs_lambda_intvl > 0 && g % S.vs_lambda_intvl == 0)
            lambda_log[ring + (size_t)((g / S.vs_lambda_intvl - 1) % log_cap)] = lambda;
    }
    if (lane == 0) {
        const VsDev &v = V[cur];
        double param = lambda;
        if (lambda <= v.lo) param = v.lo;
        else if (lambda >= v.hi) param = v.hi;
        double dlnp = v.coef[0], t = 1.0;
        for (int i = 1; i < v.order + 1; i++) {
            t *= param;
            dlnp += v.coef[i] * t;
        }
        mcmd_factor[s] = S.mcmd_k * dlnp;
    }
}

// vel_next -= moment of the atom's COM group (moment already divided by the group mass).
// ------------------------------------------------------------- integrator

// SubBox::cpy_vel_prev + update_velocities (SubBox.cpp:1427-1454) with McMD scaling of the
// work (ExtendedVMcMD::scale_force multiplies work in place).
__global__ void k_update_velocities(int n_atoms, const int *__restrict__ atom_sys, const SysDev *__restrict__ sys,
                                    const double *__restrict__ mcmd_factor, double *__restrict__ work,
                                    const float *__restrict__ mass_inv, double *__restrict__ vel,
                                    double *__restrict__ vel_next) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_atoms) return;
    const int s = atom_sys[a];
    const SysDev &S = sys[s];
    const double f = mcmd_factor[s];
    for (int q = 0; q < 3; q++) {
        const int k = 3 * a + q;
        double w = work[k];
        if (S.n_vs > 0) {
            w *= f;
            work[k] = w;
        }
        const double v = vel_next[k];
        vel[k] = v;
        vel_next[k] = v + (S.dt * -OG_FORCE_VEL * w * (double)mass_inv[a]);
    }
}

// vel_next -= moment of the atom's COM group.
__global__ void k_com_apply(int n_atoms, const int *__restrict__ atom_group, const double *__restrict__ moment,
                            const int *__restrict__ atom_sys, const int *__restrict__ sys_active,
                            double *__restrict__ v) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_atoms) return;
    const int g = atom_group[a];
    if (g < 0) return;
    if (sys_active && !sys_active[atom_sys[a]]) return;
    for (int q = 0; q < 3; q++) v[3 * a + q] -= moment[3 * g + q];
}

// Per-atom kinetic term of ThermostatScaling::apply_thermostat (Thermostat.cpp:57-73).
__global__ void k_thermo_scaling_ke(int n_atoms, const int *__restrict__ atom_sys, const SysDev *__restrict__ sys,
                                    const double *__restrict__ work, const float *__restrict__ mass,
                                    const float *__restrict__ mass_inv, const double *__restrict__ vel,
                                    double *__restrict__ tmp) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_atoms) return;
    const SysDev &S = sys[atom_sys[a]];
    double vn = 0.0;
    for (int q = 0; q < 3; q++) {
        const double vt = vel[3 * a + q] - 0.5 * (S.dt * work[3 * a + q] * OG_FORCE_VEL * (double)mass_inv[a]);
        vn += vt * vt;
    }
    tmp[a] = (double)mass[a] * vn;
}

// SubBox::update_thermostat target (SubBox.cpp:1745-1757).
// thermo[4s..4s+3] = temperature, initial temperature, heating steps, the system's first step
// (the heating ramp of SubBox.cpp:1746-1751, with the step counted from the run's start).
__device__ __forceinline__ double target_temperature(const double *thermo, int s, long long engine_step) {
    const double t0 = thermo[4 * s], tinit = thermo[4 * s + 1], heat = thermo[4 * s + 2];
    const long long step = engine_step + (long long)thermo[4 * s + 3];
    if ((double)step < heat) return tinit + ((t0 - tinit) / heat) * (double)step;
    return t0;
}

__global__ void k_thermo_scaling_apply(int n_atoms, const int *__restrict__ atom_sys, const SysDev *__restrict__ sys,
                                       const double *__restrict__ sum_ke, const double *__restrict__ thermo,
                                       const long long *__restrict__ step, const double *__restrict__ work,
                                       const float *__restrict__ mass_inv, const double *__restrict__ vel,
                                       double *__restrict__ vel_next) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_atoms) return;
    const int s = atom_sys[a];
    const SysDev &S = sys[s];
    if (S.thermostat != 1 || S.has_constraints) return;
    const double tcur = sum_ke[s] * S.temperature_coeff_thermo;
    const double tt = target_temperature(thermo, s, *step);
    const double scale = sqrt(1 + S.dt * S.tau_inv * (tt / tcur - 1));
    for (int q = 0; q < 3; q++) {
        const double vd = S.dt * -OG_FORCE_VEL * work[3 * a + q] * (double)mass_inv[a];
        vel_next[3 * a + q] = (2.0 * scale - 1.0) * vel[3 * a + q] + scale * vd;
    }
}

// SubBox::cpy_crd_prev + update_coordinates_cur (SubBox.cpp:1417-1420, 1567-1580).
__global__ void k_update_coordinates(int n_atoms, const int *__restrict__ atom_sys, const SysDev *__restrict__ sys,
                                     double *__restrict__ crd, double *__restrict__ crd_prev,
                                     const double *__restrict__ vel_next) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_atoms) return;
    const double dt = sys[atom_sys[a]].dt;
    for (int q = 0; q < 3; q++) {
        const int k = 3 * a + q;
        const double x = crd[k];
        crd_prev[k] = x;
        crd[k] = x + vel_next[k] * dt;
    }
}

// ConstraintShake::shake_pair (ConstraintShake.cpp:18-49): one analytic correction.
__global__ void k_shake_pair(int n, const int2 *__restrict__ p, const double *__restrict__ d2,
                             const int *__restrict__ psys, const SysDev *__restrict__ sys,
                             const int *__restrict__ sys_active, const float *__restrict__ mass_inv,
                             double *__restrict__ crd, const double *__restrict__ crd_prev) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int s = psys[k];
    if (sys_active && !sys_active[s]) return;
    const SysDev &S = sys[s];
    const int i = p[k].x, j = p[k].y;
    double d[3], dp[3];
    for (int q = 0; q < 3; q++) {
        d[q] = minim(crd[3 * j + q] - crd[3 * i + q], S.Lf[q], S.L_half_inv_f[q]);
        dp[q] = minim(crd_prev[3 * j + q] - crd_prev[3 * i + q], S.Lf[q], S.L_half_inv_f[q]);
    }
    const double m1 = (double)mass_inv[i], m2 = (double)mass_inv[j], m12 = m1 + m2;
    const double dsq = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    const double dsqp = dp[0] * dp[0] + dp[1] * dp[1] + dp[2] * dp[2];
    const double dip = d[0] * dp[0] + d[1] * dp[1] + d[2] * dp[2];
    const double va = m12 * m12 * dsqp, vb = m12 * dip, vc = dsq - d2[k];
    const double g = (vb - sqrt(fmax(vb * vb - vc * va, 0.0))) / va;
    for (int q = 0; q < 3; q++) {
        crd[3 * i + q] += m1 * g * dp[q];
        crd[3 * j + q] -= m2 * g * dp[q];
    }
}

// ConstraintShake::shake_trio (ConstraintShake.cpp:51-149): Newton iteration on the three
// squared distances with the cofactor inverse, until every relative residual < tol.
__global__ void k_shake_trio(int n, const int4 *__restrict__ t, const double *__restrict__ td,
                             const SysDev *__restrict__ sys, const int *__restrict__ sys_active,
                             const float *__restrict__ mass_inv, double *__restrict__ crd,
                             const double *__restrict__ crd_prev, int max_loops, double tol,
                             int *__restrict__ counters) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int s = t[k].w;
    if (sys_active && !sys_active[s]) return;
    const SysDev &S = sys[s];
    const int a1 = t[k].x, a2 = t[k].y, a3 = t[k].z;
    double d12[3], d23[3], d31[3], p12[3], p23[3], p31[3];
    for (int q = 0; q < 3; q++) {
        d12[q] = minim(crd[3 * a1 + q] - crd[3 * a2 + q], S.Lf[q], S.L_half_inv_f[q]);
        p12[q] = minim(crd_prev[3 * a1 + q] - crd_prev[3 * a2 + q], S.Lf[q], S.L_half_inv_f[q]);
        d23[q] = minim(crd[3 * a2 + q] - crd[3 * a3 + q], S.Lf[q], S.L_half_inv_f[q]);
        p23[q] = minim(crd_prev[3 * a2 + q] - crd_prev[3 * a3 + q], S.Lf[q], S.L_half_inv_f[q]);
        d31[q] = minim(crd[3 * a3 + q] - crd[3 * a1 + q], S.Lf[q], S.L_half_inv_f[q]);
        p31[q] = minim(crd_prev[3 * a3 + q] - crd_prev[3 * a1 + q], S.Lf[q], S.L_half_inv_f[q]);
    }
    const double m1 = (double)mass_inv[a1], m2 = (double)mass_inv[a2], m3 = (double)mass_inv[a3];
    const double c11 = m1 + m2, c12 = -m2, c13 = -m1;
    const double c21 = -m2, c22 = m2 + m3, c23 = -m3;
    const double c31 = -m1, c32 = -m3, c33 = m3 + m1;
    const double t0 = td[3 * k], t1 = td[3 * k + 1], t2 = td[3 * k + 2];
    double g0 = 0, g1 = 0, g2 = 0, g3 = 0, g4 = 0, g5 = 0;
    bool conv = false;
#define DOT(a, b) (a[0] * b[0] + a[1] * b[1] + a[2] * b[2])
    for (int it = 0; it < max_loops; it++) {
        for (int q = 0; q < 3; q++) {
            d12[q] += (c11 * p12[q] * g0 + c12 * p23[q] * g1 + c13 * p31[q] * g2);
            d23[q] += (c21 * p12[q] * g0 + c22 * p23[q] * g1 + c23 * p31[q] * g2);
            d31[q] += (c31 * p12[q] * g0 + c32 * p23[q] * g1 + c33 * p31[q] * g2);
        }
        const double f11 = 2.0 * c11 * DOT(d12, p12), f12 = 2.0 * c12 * DOT(d12, p23), f13 = 2.0 * c13 * DOT(d12, p31);
        const double f21 = 2.0 * c21 * DOT(d23, p12), f22 = 2.0 * c22 * DOT(d23, p23), f23 = 2.0 * c23 * DOT(d23, p31);
        const double f31 = 2.0 * c31 * DOT(d31, p12), f32 = 2.0 * c32 * DOT(d31, p23), f33 = 2.0 * c33 * DOT(d31, p31);
        const double r0 = t0 - DOT(d12, d12), r1 = t1 - DOT(d23, d23), r2 = t2 - DOT(d31, d31);
        if (fabs(r0 / t0) < tol && fabs(r1 / t1) < tol && fabs(r2 / t2) < tol) {
            conv = true;
            break;
        }
        const double det = 1.0 / (f11 * f22 * f33 + f12 * f23 * f31 + f13 * f21 * f32 - f11 * f23 * f32 -
                                  f12 * f21 * f33 - f13 * f22 * f31);
        const double b11 = f22 * f33 - f23 * f32, b12 = f32 * f13 - f33 * f12, b13 = f12 * f23 - f13 * f22;
        const double b21 = f23 * f31 - f21 * f33, b22 = f33 * f11 - f31 * f13, b23 = f13 * f21 - f11 * f23;
        const double b31 = f21 * f32 - f22 * f31, b32 = f31 * f12 - f32 * f11, b33 = f11 * f22 - f12 * f21;
        g0 = (b11 * r0 + b12 * r1 + b13 * r2) * det;
        g1 = (b21 * r0 + b22 * r1 + b23 * r2) * det;
        g2 = (b31 * r0 + b32 * r1 + b33 * r2) * det;
        g3 += g0;
        g4 += g1;
        g5 += g2;
    }
#undef DOT
    if (!conv) og_set_flag(counters, OG_FLAG_SHAKE);
    for (int q = 0; q < 3; q++) {
        crd[3 * a1 + q] += m1 * (g3 * p12[q] - g5 * p31[q]);
        crd[3 * a2 + q] += m2 * (-g3 * p12[q] + g4 * p23[q]);
        crd[3 * a3 + q] += m3 * (-g4 * p23[q] + g5 * p31[q]);
    }
}

// Per-atom KE of (vel_next + vel)/2 (start of each thermostat iteration, Thermostat.cpp:114-123).
__global__ void k_ke_mid(int n_atoms, const float *__restrict__ mass, const double *__restrict__ vel,
                         const double *__restrict__ vel_next, double *__restrict__ tmp) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_atoms) return;
    double vn = 0.0;
    for (int q = 0; q < 3; q++) {
        const double vt = (vel_next[3 * a + q] + vel[3 * a + q]) * 0.5;
        vn += vt * vt;
    }
    tmp[a] = vn * (double)mass[a];
}

// Convergence test of the thermostat loop, one thread per system (Thermostat.cpp:124-131).
// sys_active[s] stays 1 while the system still iterates; *any receives the count.  The loop
// index lives on the device (*it_ptr, advanced by k_thermo_next) so that the loop can run
// inside a graph without the host.
__global__ void k_thermo_check(int n_sys, const SysDev *__restrict__ sys, const double *__restrict__ sum_ke,
                               const double *__restrict__ thermo, const long long *__restrict__ step,
                               const int *__restrict__ it_ptr, int max_loops, double tol, int *__restrict__ sys_active,
                               int *__restrict__ any, int *__restrict__ counters) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_sys) return;
    if (!sys_active[s]) return;
    const int it = *it_ptr;
    const SysDev &S = sys[s];
    const double tcur = sum_ke[s] * S.temperature_coeff_thermo;
    const double tt = target_temperature(thermo, s, *step);
    if (it == max_loops - 1) {
        sys_active[s] = 0;
        og_set_flag(counters, OG_FLAG_THERMO);
        return;
    }
    if (fabs(tcur - tt) / tt < tol) {
        sys_active[s] = 0;
        return;
    }
    atomicAdd(any, 1);
}

// ConstraintShake::shake_quad (ConstraintShake.cpp:151-276): a centre and three partners, six
// squared distances in the pair order (0,1) (1,2) (2,0) (3,0) (2,3) (1,3) (Constraint.cpp:4),
// Newton steps solved with ConstraintObject::calc_linear_eq's elimination (Constraint.cpp:141).
__device__ int og_solve6(double a[6][6], double x[6], const double b[6]) {
    int piv[6] = {0, 1, 2, 3, 4, 5};
    for (int i = 0; i < 6; i++) {
        int idx = i;
        double mx = fabs(a[i][piv[i]]);
        for (int j = i + 1; j < 6; j++) {
            const double t = fabs(a[i][piv[j]]);
            if (t > mx) { idx = j; mx = t; }
        }
        if (idx != i) { const int t = piv[i]; piv[i] = piv[idx]; piv[idx] = t; }
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

__global__ void k_shake_quad(int n, const int4 *__restrict__ q4, const double *__restrict__ qd,
                             const int *__restrict__ qsys, const SysDev *__restrict__ sys,
                             const int *__restrict__ sys_active, const float *__restrict__ mass_inv,
                             double *__restrict__ crd, const double *__restrict__ crd_prev, int max_loops,
                             double tol, int *__restrict__ counters) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int s = qsys[k];
    if (sys_active && !sys_active[s]) return;
    const SysDev &S = sys[s];
    const int at[4] = {q4[k].x, q4[k].y, q4[k].z, q4[k].w};
    const int P[6][2] = {{0, 1}, {1, 2}, {2, 0}, {3, 0}, {2, 3}, {1, 3}};
    double mi[4];
    for (int i = 0; i < 4; i++) mi[i] = (double)mass_inv[at[i]];
    const double w[6][6] = {{mi[0] + mi[1], -mi[1], -mi[0], -mi[0], 0.0, -mi[1]},
                            {-mi[1], mi[1] + mi[2], -mi[2], 0.0, -mi[2], mi[1]},
                            {-mi[0], -mi[2], mi[2] + mi[0], mi[0], mi[2], 0.0},
                            {-mi[0], 0.0, mi[0], mi[3] + mi[0], -mi[3], -mi[3]},
                            {0.0, -mi[2], mi[2], -mi[3], mi[2] + mi[3], mi[3]},
                            {-mi[1], mi[1], 0.0, -mi[3], mi[3], mi[1] + mi[3]}};
    double dc[6][3], dp[6][3];
    for (int c = 0; c < 6; c++)
        for (int q = 0; q < 3; q++) {
            dc[c][q] = minim(crd[3 * at[P[c][0]] + q] - crd[3 * at[P[c][1]] + q], S.Lf[q], S.L_half_inv_f[q]);
            dp[c][q] = minim(crd_prev[3 * at[P[c][0]] + q] - crd_prev[3 * at[P[c][1]] + q], S.Lf[q],
                             S.L_half_inv_f[q]);
        }
    const double *d2 = qd + 6 * (size_t)k;
    double coef[6] = {0, 0, 0, 0, 0, 0}, post[6] = {0, 0, 0, 0, 0, 0};
    bool conv = false;
    for (int it = 0; it < max_loops; it++) {
        for (int c = 0; c < 6; c++) coef[c] = post[c];
        double dv[6][3];
        for (int i = 0; i < 6; i++) {
            for (int q = 0; q < 3; q++) dv[i][q] = dc[i][q];
            for (int j = 0; j < 6; j++)
                for (int q = 0; q < 3; q++) dv[i][q] += w[j][i] * dp[j][q] * coef[j];
        }
        double g[6][6];
        for (int i = 0; i < 6; i++)
            for (int j = 0; j < 6; j++)
                g[i][j] = 2.0 * w[j][i] * (dv[j][0] * dp[i][0] + dv[j][1] * dp[i][1] + dv[j][2] * dp[i][2]);
        bool ok = true;
        double sd[6];
        for (int i = 0; i < 6; i++) {
            sd[i] = d2[i] - (dv[i][0] * dv[i][0] + dv[i][1] * dv[i][1] + dv[i][2] * dv[i][2]);
            ok = ok && (fabs(sd[i] / d2[i]) < tol);
        }
        if (ok) {
            conv = true;
            break;
        }
        double rhs[6];
        for (int i = 0; i < 6; i++) {
            rhs[i] = sd[i];
            for (int j = 0; j < 6; j++) rhs[i] += g[j][i] * coef[j];
        }
        og_solve6(g, post, rhs);
    }
    if (!conv) og_set_flag(counters, OG_FLAG_SHAKE);
    for (int q = 0; q < 3; q++) {
        crd[3 * at[0] + q] += mi[0] * (coef[0] * dp[0][q] - coef[2] * dp[2][q] - coef[3] * dp[3][q]);
        crd[3 * at[1] + q] += mi[1] * (-coef[0] * dp[0][q] + coef[1] * dp[1][q] + coef[5] * dp[5][q]);
        crd[3 * at[2] + q] += mi[2] * (-coef[1] * dp[1][q] + coef[2] * dp[2][q] + coef[4] * dp[4][q]);
        crd[3 * at[3] + q] += mi[3] * (coef[3] * dp[3][q] - coef[4] * dp[4][q] - coef[5] * dp[5][q]);
    }
}

// Half-step velocities with the constraint acceleration (Thermostat.cpp:133-148).
__global__ void k_thermo_half(int n_atoms, const int *__restrict__ atom_sys, const SysDev *__restrict__ sys,
                              const int *__restrict__ sys_active, const double *__restrict__ work,
                              const float *__restrict__ mass, const float *__restrict__ mass_inv,
                              const double *__restrict__ crd, const double *__restrict__ buf_crd,
                              const double *__restrict__ vel, double *__restrict__ vel_next,
                              double *__restrict__ tmp) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_atoms) return;
    const int s = atom_sys[a];
    if (!sys_active[s]) { tmp[a] = 0.0; return; }
    const double dt = sys[s].dt, dtisq = 1.0 / (dt * dt);
    double vn = 0.0;
    for (int q = 0; q < 3; q++) {
        const int k = 3 * a + q;
        const double vd = -OG_FORCE_VEL * work[k] * (double)mass_inv[a] + (crd[k] - buf_crd[k]) * dtisq;
        vel_next[k] = vel[k] + 0.5 * dt * vd;
        vn += vel_next[k] * vel_next[k];
    }
    tmp[a] = (double)mass[a] * vn;
}

// Rescale to the target temperature (Thermostat.cpp:150-164).
__global__ void k_thermo_rescale(int n_atoms, const int *__restrict__ atom_sys, const SysDev *__restrict__ sys,
                                 const int *__restrict__ sys_active, const double *__restrict__ sum_ke,
                                 const double *__restrict__ thermo, const long long *__restrict__ step,
                                 const double *__restrict__ work, const float *__restrict__ mass_inv,
                                 const double *__restrict__ crd, const double *__restrict__ buf_crd,
                                 const double *__restrict__ vel, double *__restrict__ vel_next) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_atoms) return;
    const int s = atom_sys[a];
    if (!sys_active[s]) return;
    const SysDev &S = sys[s];
    const double dt = S.dt, dtisq = 1.0 / (dt * dt);
    const double tcur = sum_ke[s] * S.temperature_coeff_thermo;
    const double scale = sqrt(target_temperature(thermo, s, *step) / tcur);
    for (int q = 0; q < 3; q++) {
        const int k = 3 * a + q;
        const double vd = -OG_FORCE_VEL * work[k] * (double)mass_inv[a] + (crd[k] - buf_crd[k]) * dtisq;
        vel_next[k] = (2.0 * scale - 1.0) * vel[k] + scale * dt * vd;
    }
}

// crd = crd_prev + dt vel_next for still-iterating systems (Thermostat.cpp:166-170).
__global__ void k_thermo_crd(int n_atoms, const int *__restrict__ atom_sys, const SysDev *__restrict__ sys,
                             const int *__restrict__ sys_active, double *__restrict__ crd,
                             const double *__restrict__ crd_prev, const double *__restrict__ vel_next) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_atoms) return;
    const int s = atom_sys[a];
    if (!sys_active[s]) return;
    const double dt = sys[s].dt;
    for (int q = 0; q < 3; q++) crd[3 * a + q] = crd_prev[3 * a + q] + dt * vel_next[3 * a + q];
}

// The pair kernel's j lists hold while every slot is within skin of the position they were
// built from (xq_ref; null when the engine does not use them); otherwise the lists of the slot's
// system are marked stale (jl_stale[s]), with the engine-wide "some system is stale" word.  Only
// that system's lists are rebuilt, so a system's j lists, and with them the order of its FP32
// i sums, never depend on the other systems of the batch.
__device__ __forceinline__ void og_jl_check(const float4 &p, int sl, int s, const float4 *__restrict__ xq_ref,
                                            float skin2, int *__restrict__ jl_stale, int *__restrict__ counters) {
    if (!xq_ref) return;
    const float4 o = xq_ref[sl];
    const float dx = p.x - o.x, dy = p.y - o.y, dz = p.z - o.z;
    if (!(dx * dx + dy * dy + dz * dz <= skin2)) {
        jl_stale[s] = 1;
        counters[OG_CNT_JL_STALE] = 1;
    }
}

// Displacement list policy: the cell-pair list holds every pair within the list cutoff at its
// build, so it holds every pair within the interaction cutoff while no atom has moved farther
// than half the margin since (xq_build: the slot offsets at the build, null under the fixed
// schedule); past that the list is marked stale and rebuilt before the next force evaluation.
__device__ __forceinline__ void og_list_check(const float4 &p, int sl, const SysDev &S,
                                              const float4 *__restrict__ xq_build, int *__restrict__ counters) {
    if (!xq_build) return;
    const float4 o = xq_build[sl];
    const float dx = p.x - o.x, dy = p.y - o.y, dz = p.z - o.z;
    if (!(dx * dx + dy * dy + dz * dz <= S.list_trig2)) counters[OG_CNT_LIST_STALE] = 1;
}

// End of step, per atom: velocities from the constrained displacement (SubBox.cpp:1462-1481,
// only when the plain constraint path ran), MiniCell::move_atom (MiniCell.cpp:1312-1325) and the
// refreshed cell-relative float coordinate, PBC wrap (SubBox.cpp:1482-1502) and the kinetic
// term of (vel + vel_next)/2 (SubBox.cpp:1504-1516, DynamicsMode.cpp:358-372).
__global__ void k_finish(int n_atoms, const int *__restrict__ atom_sys, const SysDev *__restrict__ sys,
                         int vel_from_crd, double *__restrict__ crd, const double *__restrict__ crd_prev,
                         const double *__restrict__ vel, double *__restrict__ vel_next,
                         const int *__restrict__ atom_slot, double *__restrict__ slot_crd,
                         const double *__restrict__ cell_origin, float4 *__restrict__ xq,
                         const float *__restrict__ mass, double *__restrict__ ke, int *__restrict__ counters,
                         int *__restrict__ sys_fault, const float4 *__restrict__ xq_ref, float jl_skin2,
                         int *__restrict__ jl_stale, const float4 *__restrict__ xq_build) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n_atoms) return;
    const SysDev &S = sys[atom_sys[a]];
    const int sl = atom_slot[a], c = sl >> 3;
    double vn = 0.0, disp2 = 0.0;
    float r[3];
    for (int q = 0; q < 3; q++) {
        const int k = 3 * a + q;
        const double x = crd[k], xp = crd_prev[k];
        disp2 += (x - xp) * (x - xp);
        if (vel_from_crd && S.has_constraints && S.thermostat != 1) vel_next[k] = (x - xp) * (1.0 / S.dt);
        const double gcrd = slot_crd[3 * (size_t)sl + q] + (x - xp);
        slot_crd[3 * (size_t)sl + q] = gcrd;
        r[q] = (float)(gcrd - cell_origin[3 * c + q]);
        double xw = x;
        if (xw >= (double)S.upperf[q]) xw -= (double)S.Lf[q];
        else if (xw < (double)S.lowerf[q]) xw += (double)S.Lf[q];
        crd[k] = xw;
        const double vj = (vel[k] + vel_next[k]) * 0.5;
        vn += vj * vj;
    }
    float4 p = xq[sl];
    p.x = r[0];
    p.y = r[1];
    p.z = r[2];
    xq[sl] = p;
    og_jl_check(p, sl, atom_sys[a], xq_ref, jl_skin2, jl_stale, counters);
    og_list_check(p, sl, S, xq_build, counters);
    ke[a] = vn * (double)mass[a];
    if (!(disp2 <= S.max_step_disp2)) {  // also catches NaN
        og_set_flag(counters, OG_FLAG_DISPLACEMENT);
        atomicOr(&sys_fault[atom_sys[a]], OG_FLAG_DISPLACEMENT);
    }
}

// Slot coordinates/charges/types after a list rebuild (cuda_setup.cu:364-402 roles).
__global__ void k_slot_refresh(const int *__restrict__ counters, int slots_cap, const int *__restrict__ slot_atom,
                               const double *__restrict__ slot_crd, const double *__restrict__ cell_origin,
                               const float *__restrict__ charge_f, const int *__restrict__ atom_type,
                               float4 *__restrict__ xq, int *__restrict__ slot_type) {
    int sl = blockIdx.x * blockDim.x + threadIdx.x;
    const int n_slots = counters[OG_CNT_N_CELLS] * OG_CELL;
    if (sl >= n_slots || sl >= slots_cap) return;
    const int c = sl >> 3, a = slot_atom[sl];
    float4 p;
    p.x = (float)(slot_crd[3 * (size_t)sl] - cell_origin[3 * c]);
    p.y = (float)(slot_crd[3 * (size_t)sl + 1] - cell_origin[3 * c + 1]);
    p.z = (float)(slot_crd[3 * (size_t)sl + 2] - cell_origin[3 * c + 2]);
    p.w = a >= 0 ? charge_f[a] : 0.0f;
    xq[sl] = p;
    slot_type[sl] = a >= 0 ? atom_type[a] : 0;
}

// Final per-system energies of a step (DynamicsMode::gather_energies + cal_kinetic_energy),
// appended to the trace ring when enabled.
__global__ void k_energies(int n_sys, const SysDev *__restrict__ sys, const double *__restrict__ sys_acc,
                           const double *__restrict__ mcmd_factor, double *__restrict__ energies,
                           double *__restrict__ trace, int trace_cap, long long *__restrict__ trace_count) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_sys) return;
    const SysDev &S = sys[s];
    const double *acc = sys_acc + OG_ACC_SIZE * s;
    double *e = energies + OG_N_ENERGY * s;
    e[OG_E_VDW] = acc[OG_ACC_VDW];
    e[OG_E_ELE] = acc[OG_ACC_ELE] + acc[OG_ACC_EXCESS] + S.self_energy;
    e[OG_E_BOND] = acc[OG_ACC_BOND];
    e[OG_E_ANGLE] = acc[OG_ACC_ANGLE];
    e[OG_E_TORSION] = acc[OG_ACC_TORSION];
    e[OG_E_IMPROPER] = acc[OG_ACC_IMPRO];
    e[OG_E_VDW14] = acc[OG_ACC_VDW14];
    e[OG_E_ELE14] = acc[OG_ACC_ELE14];
    e[OG_E_POTENTIAL] = e[OG_E_VDW] + e[OG_E_ELE] + e[OG_E_BOND] + e[OG_E_ANGLE] + e[OG_E_TORSION] +
                        e[OG_E_IMPROPER] + e[OG_E_VDW14] + e[OG_E_ELE14];
    e[OG_E_KINETIC] = acc[OG_ACC_KIN] * OG_KINETIC_COEFF;
    e[OG_E_TEMPERATURE] = e[OG_E_KINETIC] * S.temperature_coeff_dyn;
    e[OG_E_TOTAL] = e[OG_E_POTENTIAL] + e[OG_E_KINETIC];
    e[OG_E_ELE_EXCESS] = acc[OG_ACC_EXCESS];
    e[OG_E_ELE_SELF] = S.self_energy;
    e[OG_E_MCMD_FACTOR] = mcmd_factor[s];
    if (trace && trace_cap > 0) {
        const long long row = *trace_count % trace_cap;
        for (int q = 0; q < OG_N_ENERGY; q++) trace[(row * n_sys + s) * OG_N_ENERGY + q] = e[q];
    }
}

// og_put_state: continue the trajectory from host coordinates without re-enumerating pairs
// (the role of cuda_memcpy_htod_crd + kernel_set_crd, cuda_setup.cu:124-136, 380-402): the
// grid copy moves by the minimum-image displacement, as MiniCell::move_atom does.
__global__ void k_put_state(int n_atoms, int atom0, const int *__restrict__ atom_sys,
                            const SysDev *__restrict__ sys, const double *__restrict__ new_crd,
                            const double *__restrict__ new_vel, double *__restrict__ crd,
                            double *__restrict__ vel_next, const int *__restrict__ atom_slot,
                            double *__restrict__ slot_crd, const double *__restrict__ cell_origin,
                            float4 *__restrict__ xq, const float4 *__restrict__ xq_ref, float jl_skin2,
                            int *__restrict__ jl_stale, const float4 *__restrict__ xq_build,
                            int *__restrict__ counters) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_atoms) return;
    const int a = atom0 + i;
    const SysDev &S = sys[atom_sys[a]];
    const int sl = atom_slot[a], c = sl >> 3;
    float4 p = xq[sl];
    float r[3];
    for (int q = 0; q < 3; q++) {
        if (new_crd) {
            const double x = new_crd[3 * i + q];
            double d = x - crd[3 * a + q];
            d -= S.L[q] * nearbyint(d / S.L[q]);
            const double g = slot_crd[3 * (size_t)sl + q] + d;
            slot_crd[3 * (size_t)sl + q] = g;
            r[q] = (float)(g - cell_origin[3 * c + q]);
            // held in the box as every step end holds it (SubBox.cpp:1482-1502), so that a list
            // built from it puts the atom in the column of its own grid coordinate
            double xw = x;
            if (xw >= (double)S.upperf[q]) xw -= (double)S.Lf[q];
            else if (xw < (double)S.lowerf[q]) xw += (double)S.Lf[q];
            crd[3 * a + q] = xw;
        }
        if (new_vel) vel_next[3 * a + q] = new_vel[3 * i + q];
    }
    if (new_crd) {
        p.x = r[0];
        p.y = r[1];
        p.z = r[2];
        xq[sl] = p;
        og_jl_check(p, sl, atom_sys[a], xq_ref, jl_skin2, jl_stale, counters);
        og_list_check(p, sl, S, xq_build, counters);
    }
}

// Displacement list policy inside a captured graph: the IF node around the list build runs its
// body when the list is stale, unless a system has faulted in this call (the call is undone;
// no list is built from its non-finite or runaway coordinates).
__global__ void k_list_cond(const int *__restrict__ counters, cudaGraphConditionalHandle cond) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const bool fault = (counters[OG_CNT_FLAGS] & (OG_FLAG_BAD_COORD | OG_FLAG_COLUMN_CAPACITY |
                                                      OG_FLAG_DISPLACEMENT)) != 0;
        cudaGraphSetConditional(cond, (counters[OG_CNT_LIST_STALE] && !fault) ? 1u : 0u);
    }
}

// Advances the thermostat loop index and clears the "still iterating" count for the next
// pass.  Inside a graph (use_cond) it also sets the loop's conditional node: another pass only
// while some system still iterates and fewer than max_loops passes have run, so the device-side
// loop ends after max_loops passes at most, whatever the data.
__global__ void k_thermo_next(int *__restrict__ any, int *__restrict__ it, int max_loops,
                              cudaGraphConditionalHandle cond, int use_cond) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int next = *it + 1;
    const int still = *any;
    *it = next;
    *any = 0;
    if (use_cond) cudaGraphSetConditional(cond, (still != 0 && next < max_loops) ? 1u : 0u);
}

__global__ void k_trace_advance(long long *trace_count, long long *step) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        *trace_count += 1;
        *step += 1;
    }
}


// Trajectory frames (DynamicsMode::sub_output, DynamicsMode.cpp:264-300), captured at the end
// of step g for the frame labelled k = g + 1 when k is a multiple of the system's interval: the
// coordinates at which step g's forces were computed (SubBox::crd_prev, which is what the
// reference writes), rounded to FP32 as WriteTrrPresto / WriteTrrGromacs store them, and step
// g's energies.  One thread per (group atom, system entry); frame k sits in ring slot
// (k / interval - 1) mod frames.  Launched before the step counter advances.
__global__ void k_capture_frames(int n_entries, const int *__restrict__ tr_atom, const int *__restrict__ tr_sys,
                                 const int *__restrict__ tr_idx, const SysDev *__restrict__ sys,
                                 const long long *__restrict__ step, const double *__restrict__ crd_prev,
                                 const double *__restrict__ energies, float *__restrict__ frames,
                                 double *__restrict__ frame_ene) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_entries) return;
    const int s = tr_sys[i];
    const SysDev &S = sys[s];
    const long long k = *step + S.first_step + 1;
    if (k % S.tr_interval != 0) return;
    const long long slot = (k / S.tr_interval - 1) % S.tr_frames;
    const int a = tr_atom[i], j = tr_idx[i];
    float *f = frames + S.tr_crd_base + (slot * S.tr_n + j) * 3;
    f[0] = (float)crd_prev[3 * a];
    f[1] = (float)crd_prev[3 * a + 1];
    f[2] = (float)crd_prev[3 * a + 2];
    if (j == 0) {
        double *e = frame_ene + S.tr_ene_base + slot * OG_N_ENERGY;
        for (int q = 0; q < OG_N_ENERGY; q++) e[q] = energies[OG_N_ENERGY * s + q];
    }
}

}  // namespace og
