// og_engine.cu -- host side of the engine and the C ABI declared in include/omegagene_b200.h.
//
// Owns every device buffer of a batch of systems, computes the MiniCell geometry on the host
// with the reference's float arithmetic (MiniCell.cpp:221-290, 1279-1303), and sequences the
// kernels of one DynamicsModePresto step (DynamicsMode.cpp:468-560) on one CUDA stream.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/omegagene_b200.h"
#include "og_internal.cuh"

namespace og {
// og_grid.cu
__global__ void k_assign_columns(const SysDev *, const int *, const double *, int, int *, unsigned long long *,
                                 int *, int *, int *);
__global__ void k_scan_columns(const int *, int, int *, int *, int *, int *, const int *, int, int *);
__global__ void k_scatter_columns(const int *, const unsigned long long *, int, const int *, int *,
                                  unsigned long long *);
__global__ void k_sort_columns(const int *, const int *, const int *, const int *, const unsigned long long *,
                               const SysDev *, const double *, int *, double *, int *, int *, int *, int *, int *);
__global__ void k_cell_info(const int *, int, const int *, const int *, const int *, const SysDev *, const double *,
                            const int *, double *, float2 *, int2 *, unsigned char *, int *, int *);
__global__ void k_count_pairs(const int *, int, int, const int *, const int *, const SysDev *, const int *,
                              const int *, const int *, const float2 *, const int2 *, const int *, const int *,
                              const int *, int *);
__global__ void k_fill_pairs(int *, int, int, long long, const int *, const int *, const SysDev *, const int *,
                             const int *, const int *, const float2 *, const int2 *, const int *, const int *,
                             const int *, const long long *, int2 *);
__global__ void k_pair_records(const int *, long long, const int *, const SysDev *, const int *, const int2 *,
                               const unsigned char *, const int *, const int *, const int *, const int *, const int *,
                               const double *, unsigned long long *, float4 *);
__global__ void k_cell_excl(const int *, int, const int *, const int *, const int *, const int *, int *);
__global__ void k_pair_heads(int *, int, int, long long, const long long *, int *);
template <typename TI>
__global__ void k_scan_block(const TI *, long long *, long long, long long *);
__global__ void k_scan_add(long long *, long long, const long long *);
// og_pair.cu
template <bool VIR, int MINB>
__global__ void k_pair_ljzd(const int *, const int *, const SysDev *, const float4 *, const float4 *, const int *,
                            const int *, const float4 *, const int2 *, const unsigned long long *, const float2 *,
                            unsigned long long *, double *, long long);
template <bool VIR, int MINB>
__global__ void k_pair_ljzd_jm(const int *, const int *, const SysDev *, const float4 *, const float4 *, const int *,
                               const int *, const float4 *, const int2 *, const unsigned long long *, const float2 *,
                               unsigned long long *, double *, long long);
template <bool VIR, bool ENE, int MINB, int NT, bool GEN>
__global__ void k_pair_ljzd_jq(const int *, const int *, const SysDev *, const float4 *, const float4 *, const int *,
                               const int *, const float4 *, const int2 *, const unsigned long long *, const float2 *,
                               unsigned long long *, double *, long long, const EleDev *, const float2 *);
template <bool VIR, bool ENE, int MINB>
__global__ void k_pair_ljzd_jm2(const int *, const int *, const SysDev *, const float4 *, const float4 *, const int *,
                                const int *, const float4 *, const int2 *, const unsigned long long *, const float2 *,
                                unsigned long long *, double *, long long);
template <bool VIR, bool ENE, int MINB, int NT, bool GEN>
__global__ void k_pair_ljzd_jl(int *, const int *, const SysDev *, const float4 *, const int *, const int *,
                               const float4 *, const int2 *, const int2 *, const int *, const float2 *,
                               unsigned long long *, double *, const EleDev *, const float2 *, int *, int);
template <bool VIR>
__global__ void k_pair_f64(const int *, const int *, const SysDev *, const double *, const int *, const int *,
                           const double *, const int *, const int2 *, const unsigned long long *, const double2 *,
                           long long, unsigned long long *, double *);
template <int NT>
__global__ void k_jl_build(int *, const int *, const SysDev *, const float4 *, const float4 *, const int *,
                           const float4 *, const unsigned long long *, long long, float, int2 *, int *, float4 *,
                           const int *);
__global__ void k_cell_bbox(const int *, int, const float4 *, const unsigned char *, float4 *);
// og_integrate.cu
__global__ void k_excess(int, const int2 *, const int *, const SysDev *, const EleDev *, const double *,
                         const double *, const int *, unsigned long long *, double *, double *);
__global__ void k_bonds(int, const int2 *, const double2 *, const int *, const SysDev *, const double *, const int *,
                        unsigned long long *, double *);
__global__ void k_angles(int, const int4 *, const double2 *, const SysDev *, const double *, const int *,
                         unsigned long long *, double *);
__global__ void k_atom_virial(int, const int *, const unsigned long long *, const float4 *, const double *, double *);
__global__ void k_collect_slots(const int *, int, const int *, unsigned long long *, double *);
template <int NV>
__global__ void k_part(const double *, int, int, const int *, int, double *);
__global__ void k_part_momentum(const int *, const int *, const float *, const double *, const int *, const int *,
                                int, double *);
template <int NV>
__global__ void k_part_final(const double *, int, double *, int, int, const float *, int);
__global__ void k_vmcmd(int, const SysDev *, const VsDev *, const double *, const long long *, int, int *, unsigned *,
                        int *, double *, int, double *);
__global__ void k_update_velocities(int, const int *, const SysDev *, const double *, double *, const float *,
                                    double *, double *);
__global__ void k_com_apply(int, const int *, const double *, const int *, const int *, double *);
__global__ void k_thermo_scaling_ke(int, const int *, const SysDev *, const double *, const float *, const float *,
                                    const double *, double *);
__global__ void k_thermo_scaling_apply(int, const int *, const SysDev *, const double *, const double *,
                                       const long long *, const double *, const float *, const double *, double *);
__global__ void k_update_coordinates(int, const int *, const SysDev *, double *, double *, const double *);
__global__ void k_shake_pair(int, const int2 *, const double *, const int *, const SysDev *, const int *,
                             const float *, double *, const double *);
__global__ void k_shake_trio(int, const int4 *, const double *, const SysDev *, const int *, const float *, double *,
                             const double *, int, double, int *);
__global__ void k_ke_mid(int, const float *, const double *, const double *, double *);
__global__ void k_thermo_check(int, const SysDev *, const double *, const double *, const long long *, const int *,
                               int, double, int *, int *, int *);
__global__ void k_thermo_next(int *, int *, int, cudaGraphConditionalHandle, int);
__global__ void k_thermo_half(int, const int *, const SysDev *, const int *, const double *, const float *,
                              const float *, const double *, const double *, const double *, double *, double *);
__global__ void k_thermo_rescale(int, const int *, const SysDev *, const int *, const double *, const double *,
                                 const long long *, const double *, const float *, const double *, const double *,
                                 const double *, double *);
__global__ void k_thermo_crd(int, const int *, const SysDev *, const int *, double *, const double *,
                             const double *);
__global__ void k_dihedrals(int, const int4 *, const double4 *, const int *, const SysDev *, const double *, const int *,
                            unsigned long long *, double *);
__global__ void k_nb14(int, const int2 *, const int2 *, const double2 *, const int *, const SysDev *, const double *,
                       const float *, const float2 *, const int *, unsigned long long *, double *);
__global__ void k_shake_quad(int, const int4 *, const double *, const int *, const SysDev *, const int *, const float *,
                             double *, const double *, int, double, int *);
__global__ void k_finish(int, const int *, const SysDev *, int, double *, const double *, const double *, double *,
                         const int *, double *, const double *, float4 *, const float *, double *, int *, int *,
                         const float4 *, float, int *, const float4 *);
__global__ void k_slot_refresh(const int *, int, const int *, const double *, const double *, const float *,
                               const int *, float4 *, int *);
__global__ void k_energies(int, const SysDev *, const double *, const double *, double *, double *, int,
                           long long *);
__global__ void k_trace_advance(long long *, long long *);
__global__ void k_capture_frames(int, const int *, const int *, const int *, const SysDev *, const long long *,
                                 const double *, const double *, float *, double *);
__global__ void k_put_state(int, int, const int *, const SysDev *, const double *, const double *, double *, double *,
                            const int *, double *, const double *, float4 *, const float4 *, float, int *,
                            const float4 *, int *);
__global__ void k_list_cond(const int *, cudaGraphConditionalHandle);

__global__ void k_fill_int(int *p, long long n, int v) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}
__global__ void k_copy_double(double *dst, const double *src, long long n) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i];
}
}  // namespace og

using namespace og;

// The pair variant over j lists, and the default displacement (A) after which its lists are
// rebuilt (OG_JL_SKIN in the environment overrides it, 0.05-2 A).
#define OG_JL_VARIANT 10
#define OG_JL_BUILDS_PER_STEP 0.5  // j-list builds per step charged to variant 10 by the autotuner
#define OG_JL_SKIN 0.35f

namespace {

struct HostSystem {
    og_system_desc d;  // pointers below refer to the owned vectors
    std::vector<double> crd, vel, charge, mass, lj6, lj12, spd, std_, bk, br0, ak, at0, mcoef;
    std::vector<int32_t> type, excl, sp, st, bond, angle, gstart, gatoms;
    SysDev dev;
    int n_excess = 0;
    std::vector<int32_t> excess;  // pairs (i<j) in MmSystem::set_excess_pairs order, local ids
    std::vector<int32_t> xs, xl;  // exclusion partners per atom (CSR, insertion order), local ids
    std::vector<int32_t> tq, tov, tsym, iq, iov, isym, p14, t14, qa;  // dihedrals, 1-4 pairs, SHAKE quads
    std::vector<double> tene, tph, iene, iph, cv14, ce14, qd;
    std::vector<VsDev> vstates;   // V-McMD states (one for the one-state mcmd_* form)
    std::vector<uint32_t> mt;     // generator at the system's first step ([OG_MT_WORDS])
    std::vector<int32_t> tr_group;  // trajectory group (local atom ids), og_set_trajectory
    int tr_interval = 0;
    std::vector<double> hcut, hlam;  // HPS tables [n_lj_types^2]
    EleDev ele{};                    // electrostatics / nonbond model
    int d_free = 0;
};

// Host side of one system's trajectory frames: frames moved off the device ring, not yet taken.
// Frame k (1-based) is labelled step k * interval; next_k is the first frame still on the ring.
struct TrLog {
    long long next_k = 1;
    std::vector<long long> step;
    std::vector<float> crd;    // [frames][group][3]
    std::vector<double> ene;   // [frames][OG_N_ENERGY]
    size_t head = 0;           // frames before the head were taken
};

// Host side of one system's V-McMD logs: entries moved off the device ring and not yet taken.
// Entry k (1-based) of a log belongs to step k * interval; next_k is the first entry still on
// the ring only.
struct VmLog {
    long long vs_next_k = 1, lam_next_k = 1;
    std::vector<long long> vs_step, lam_step;
    std::vector<int32_t> vs;
    std::vector<double> lam;
    size_t vs_head = 0, lam_head = 0;  // entries before the head were taken
};

template <class T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
};

}  // namespace

struct og_engine {
    int device = 0;
    int poison = -1;  // OG_DEBUG_POISON: byte every new device buffer is filled with (-1: none)
    cudaStream_t stream = nullptr;
    std::string err;
    bool finalized = false;
    std::vector<HostSystem> sys;
    // sizes
    int n_sys = 0, n_atoms = 0, n_cols = 0, n_uni = 0, cells_cap = 0, slots_cap = 0, nnc = 1, intvl = 1;
    long long pair_cap = 0;
    int n_excess = 0, n_bonds = 0, n_angles = 0, n_spair = 0, n_strio = 0, n_groups = 0;
    int shake_max_loops = 1000, thermo_max_loops = 100;
    double shake_tol = 1e-7, thermo_tol = 1e-5;
    bool any_groups = false, any_thermo_free = false, any_thermo_cons = false, any_plain_cons = false;
    bool any_bonds = false, any_angles = false, any_mcmd = false;
    long long host_step = 0;
    // device buffers
    SysDev *d_sys = nullptr;
    int *d_counters = nullptr;
    long long *d_step = nullptr, *d_trace_count = nullptr;
    double *d_crd = nullptr, *d_crd_prev = nullptr, *d_vel = nullptr, *d_vel_next = nullptr, *d_work = nullptr,
           *d_buf_crd = nullptr, *d_charge = nullptr, *d_ke = nullptr, *d_vir_atom = nullptr;
    float *d_charge_f = nullptr, *d_mass = nullptr, *d_mass_inv = nullptr;
    int *d_atom_type = nullptr, *d_atom_sys = nullptr, *d_atom_col = nullptr, *d_atom_slot = nullptr,
        *d_atom_group = nullptr;
    unsigned long long *d_atom_key = nullptr, *d_col_keys = nullptr;
    int *d_col_count = nullptr, *d_col_fill = nullptr, *d_col_atom_start = nullptr, *d_col_cell_start = nullptr,
        *d_col_head_cell = nullptr, *d_col_sys = nullptr, *d_sys_col_base = nullptr, *d_sys_cell_base = nullptr;
    int *d_cell_col = nullptr, *d_cell_sys = nullptr, *d_cp_head = nullptr;
    double *d_cell_origin = nullptr, *d_cell_acc = nullptr;
    float2 *d_cell_zr = nullptr;
    int2 *d_cell_uni = nullptr;
    unsigned char *d_cell_valid = nullptr;
    int *d_slot_atom = nullptr, *d_slot_type = nullptr;
    double *d_slot_crd = nullptr;
    float4 *d_xq = nullptr;
    // j lists of the pair variant OG_JL_VARIANT: entries (8 per cell-pair record), per-cell
    // counts, and the slot positions they were built from
    int2 *d_jl = nullptr;
    int *d_jl_count = nullptr;
    float4 *d_xq_ref = nullptr;
    int *d_jl_stale = nullptr;   // per system: its j lists must be rebuilt before the next pair launch
    // cell-pair list schedule: OG_LIST_FIXED (the reference's, every nsgrid_update_intvl steps) or
    // OG_LIST_DISPLACEMENT (whenever an atom has moved half the list margin since the last build)
    int list_policy = OG_LIST_FIXED;
    bool pair_only = false;  // og_set_pair_only: the pair LJ + ZD terms alone (no excluded-pair term)
    float4 *d_xq_build = nullptr;  // slot offsets at the last list build (displacement policy only)
    // launch accounting of the conditional list build inside graph replays: the kernels of one
    // build (not counted per replay), builds launched kernel by kernel in the current og_step, and
    // the list-build counter as last read from the device
    long long cond_build_kernels = 0, host_cond_builds = 0, builds_seen = 0;
    float jl_skin = OG_JL_SKIN;
    unsigned long long *d_frc = nullptr;
    int *d_uni_lo = nullptr, *d_uni_hi = nullptr;
    int *d_count = nullptr;
    long long *d_offset = nullptr;        // 64-bit exclusive scan of d_count (pair list offsets)
    std::vector<long long *> d_scan_tmp;  // per level: sums, scanned sums
    std::vector<long long> scan_len;
    int2 *d_cp_c2img = nullptr;
    unsigned long long *d_cp_mask = nullptr;
    float4 *d_cp_shift = nullptr;  // pair-kernel record: FP64-formed shift + cell2
    float4 *d_bbox = nullptr;      // per-cell bounding boxes (2 per cell)
    int *d_excl_start = nullptr, *d_excl_list = nullptr;
    int2 *d_excess = nullptr;
    int *d_excess_sys = nullptr;
    double *d_e_exc = nullptr, *d_vir_exc = nullptr;
    int2 *d_bond = nullptr;
    int *d_bond_sys = nullptr;
    double2 *d_bond_kr = nullptr;
    double *d_e_bond = nullptr;
    int4 *d_angle = nullptr;
    double2 *d_angle_kt = nullptr;
    double *d_e_angle = nullptr;
    int4 *d_tors = nullptr, *d_impro = nullptr, *d_squad = nullptr;
    double4 *d_tors_p = nullptr, *d_impro_p = nullptr;
    int *d_tors_sys = nullptr, *d_impro_sys = nullptr, *d_nb14_sys = nullptr, *d_squad_sys = nullptr;
    double *d_e_tors = nullptr, *d_e_impro = nullptr, *d_e_nb14 = nullptr, *d_squad_d2 = nullptr;
    int2 *d_nb14 = nullptr, *d_nb14_t = nullptr;
    double2 *d_nb14_c = nullptr;
    int n_tors = 0, n_impro = 0, n_nb14 = 0, n_squad = 0;
    int *d_seg_tors = nullptr, *d_seg_impro = nullptr, *d_seg_nb14 = nullptr;
    int mc_tors = 1, mc_impro = 1, mc_nb14 = 1;
    int2 *d_spair = nullptr;
    int *d_spair_sys = nullptr;
    double *d_spair_d2 = nullptr;
    int4 *d_strio = nullptr;
    double *d_strio_d2 = nullptr;
    int *d_grp_start = nullptr, *d_grp_atoms = nullptr, *d_grp_sys = nullptr;
    float *d_grp_mass_inv = nullptr;
    double *d_moment = nullptr;
    float2 *d_lj = nullptr;
    double2 *d_lj64 = nullptr;  // FP64 C6/C12 of the validation variant OG_PAIR_VARIANT_F64 (else null)
    double *d_sys_acc = nullptr, *d_mcmd = nullptr, *d_energies = nullptr, *d_thermo = nullptr,
           *d_sum_tmp = nullptr;
    int *d_mask_plain = nullptr, *d_mask_thermo = nullptr, *d_active = nullptr, *d_any = nullptr,
        *d_thermo_it = nullptr;
    int *d_sys_fault = nullptr;           // per system: OG_FLAG_BAD_COORD / OG_FLAG_COLUMN_CAPACITY
    long long *d_snap_ctr = nullptr;      // step and trace counters at the start of og_step
    int *d_cell_excl = nullptr;           // per cell: excluded-partner (cell, bit) row, OG_CELL_EXCL ints
    std::vector<int32_t> faults;          // per-system fault bits of the last failed call
    // CUDA graph of one list interval (a rebuild step + intvl-1 steps), replayed by og_step
    cudaStream_t side = nullptr;       // captures the thermostat loop body
    cudaGraphExec_t graph_exec = nullptr;
    bool use_graphs = true, capturing = false;
    std::string graph_note;           // why graph capture turned graphs off, if it did
    long long graph_kernels = 0;      // kernel launches one replay stands for
    long long graph_replays = 0;
    // one step with energies, replayed by og_step_async under the displacement list policy
    // (whose rebuilds are conditional nodes, so the graph holds at any step)
    cudaGraphExec_t graph1_exec = nullptr;
    long long graph1_kernels = 0;
    bool graph1_failed = false;       // capture failed once: single steps run kernel by kernel
    // segment bases for the two-level reductions and their chunk counts
    int *d_seg_atoms = nullptr, *d_seg_exc = nullptr, *d_seg_bond = nullptr, *d_seg_angle = nullptr;
    int mc_atoms = 1, mc_cells = 1, mc_exc = 1, mc_bond = 1, mc_angle = 1, mc_grp = 1;
    double *d_part = nullptr;
    // trace
    double *d_trace = nullptr;
    int trace_cap = 0;
    // snapshot for capacity retries
    double *d_snap = nullptr;
    // host pinned
    int *h_pinned = nullptr;
    // stats
    long long launches = 0;
    cudaEvent_t ev_pair0 = nullptr, ev_pair1 = nullptr, ev_step0 = nullptr, ev_step1 = nullptr;
    std::vector<cudaEvent_t> pev0, pev1;  // per pair-kernel launch of one og_step
    int pev_used = 0;
    double *d_stage = nullptr;            // og_put_state staging (6 doubles per atom)
    double pair_ms = 0.0, step_ms = 0.0;
    int pair_variant = 0;
    int fixed_variant = -1;  // og_set_tuning: variant chosen by the caller, -1 = autotune
    double variant_ms[OG_N_PAIR_VARIANTS] = {};
    int timing = 0;  // 1: step + per-pair-kernel events (kernel by kernel); 2: step events only
    std::vector<void *> allocs;
    std::vector<size_t> alloc_bytes;          // size of each entry of allocs
    size_t bytes_held = 0, bytes_peak = 0;    // device bytes held by the engine now / at most
    // V-McMD: state table, per-system current state, per-slot generators and log rings
    VsDev *d_vstates = nullptr;
    int *d_vs_cur = nullptr, *d_vs_log = nullptr, *d_vm_snap_cur = nullptr;
    unsigned *d_mt = nullptr, *d_vm_snap_mt = nullptr;
    double *d_lambda_log = nullptr;
    int n_vm = 0, vm_log_cap = 0, vm_advance = 0;
    std::vector<int> vm_sys;      // system of each slot
    std::vector<VmLog> vm;        // per slot
    long long log_limit = 0;       // host_step up to which no ring overflows before a drain
    // trajectory frames: entries (group atom, system, index in group), rings, host side
    int *d_tr_atom = nullptr, *d_tr_sys = nullptr, *d_tr_idx = nullptr;
    float *d_frames = nullptr;
    double *d_frame_ene = nullptr;
    int n_tr = 0, n_tr_entries = 0;
    std::vector<int> tr_sys;      // system of each trajectory slot
    std::vector<TrLog> tr;        // per slot
    // electrostatics / nonbond models (EleDev per system) and HPS tables (aligned with d_lj)
    EleDev *d_ele = nullptr;
    float2 *d_hps = nullptr;
    bool any_gen = false;         // some system needs the generic pair-kernel path
};

namespace {

og_status fail(og_engine *e, og_status s, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (e) e->err = buf;
    return s;
}

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t _e = (call);                                                                   \
        if (_e != cudaSuccess)                                                                     \
            return fail(e, _e == cudaErrorMemoryAllocation ? OG_ERR_NOMEM : OG_ERR_CUDA, "%s: %s (%s:%d)", \
                        #call, cudaGetErrorString(_e), __FILE__, __LINE__);                        \
    } while (0)

#define LAUNCH_CHECK()                                                                             \
    do {                                                                                           \
        e->launches++;                                                                             \
        cudaError_t _e = cudaGetLastError();                                                       \
        if (_e != cudaSuccess)                                                                     \
            return fail(e, OG_ERR_CUDA, "kernel launch: %s (%s:%d)", cudaGetErrorString(_e), __FILE__, __LINE__); \
    } while (0)

// Device memory comes from one stream-ordered pool per device that keeps what engines free
// (release threshold = unlimited): a serving loop that re-creates engines for every new batch
// then reuses the same memory without returning it to the driver and mapping it again, and an
// engine's teardown does not wait on the whole device.  og_release_pool_memory gives the
// reserve back.
std::mutex g_pool_mu;
cudaMemPool_t g_pool[256] = {};

cudaError_t engine_pool(int device, cudaMemPool_t *out) {
    if (device < 0 || device >= 256) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pool[device]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        cudaError_t r = cudaMemPoolCreate(&pool, &props);
        if (r != cudaSuccess) return r;
        uint64_t keep = UINT64_MAX;
        r = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (r != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return r;
        }
        g_pool[device] = pool;
    }
    *out = g_pool[device];
    return cudaSuccess;
}

template <class T>
og_status dalloc(og_engine *e, T **p, size_t n) {
    if (n == 0) n = 1;
    void *q = nullptr;
    cudaMemPool_t pool = nullptr;
    cudaError_t r = engine_pool(e->device, &pool);
    if (r == cudaSuccess) r = cudaMallocFromPoolAsync(&q, n * sizeof(T), pool, e->stream);
    if (r != cudaSuccess)
        return fail(e, OG_ERR_NOMEM, "device allocation (%zu bytes): %s", n * sizeof(T), cudaGetErrorString(r));
    // debug: a buffer that a kernel reads before anything wrote it then shows up as a result
    // that depends on the fill byte (two runs with different bytes must agree bit for bit)
    if (e->poison >= 0 && (r = cudaMemsetAsync(q, e->poison, n * sizeof(T), e->stream)) != cudaSuccess)
        return fail(e, OG_ERR_CUDA, "poison fill: %s", cudaGetErrorString(r));
    e->allocs.push_back(q);
    e->alloc_bytes.push_back(n * sizeof(T));
    e->bytes_held += n * sizeof(T);
    e->bytes_peak = std::max(e->bytes_peak, e->bytes_held);
    *p = (T *)q;
    return OG_OK;
}

void dfree(og_engine *e, void *p) {
    if (!p) return;
    for (size_t i = 0; i < e->allocs.size(); i++)
        if (e->allocs[i] == p) {
            e->bytes_held -= e->alloc_bytes[i];
            e->allocs.erase(e->allocs.begin() + i);
            e->alloc_bytes.erase(e->alloc_bytes.begin() + i);
            break;
        }
    cudaFreeAsync(p, e->stream);
}

template <class T>
og_status upload(og_engine *e, T **p, const std::vector<T> &v) {
    og_status s = dalloc(e, p, v.size());
    if (s) return s;
    if (!v.empty()) CK(cudaMemcpyAsync(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, e->stream));
    return OG_OK;
}

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// ---------------------------------------------------------- host geometry

// PBC::set_pbc (PBC.cpp:19-41) + MiniCell geometry (MiniCell.cpp:221-290, 1279-1303).
og_status setup_geometry(og_engine *e, HostSystem &h) {
    SysDev &S = h.dev;
    const og_system_desc &d = h.d;
    float L[3] = {(float)d.pbc_val[0], (float)d.pbc_val[4], (float)d.pbc_val[8]};
    for (int i = 0; i < 3; i++) {
        if (!(L[i] > 0.0f)) return fail(e, OG_ERR_INVALID, "box length %d must be positive", i);
        float Lh = (float)((double)L[i] * 0.5);
        S.Lf[i] = L[i];
        S.L_half_inv_f[i] = (float)(1.0 / (double)Lh);
        S.lowerf[i] = (float)(d.pbc_val[9 + i] - (double)Lh);
        S.upperf[i] = S.lowerf[i] + L[i];
        S.L[i] = (double)L[i];
        S.lower[i] = (double)S.lowerf[i];
        S.upper[i] = (double)S.upperf[i];
    }
    const float cp = (float)d.nsgrid_cutoff;
    const float cph = (float)((double)cp * 0.5);
    S.cutoff_pair2 = cp * cp;
    S.n_uni_z = (int)(L[2] / cph);
    if (S.n_uni_z < 1) return fail(e, OG_ERR_INVALID, "box z length below half the pair-list cutoff");
    S.L_z_uni = L[2] / (float)S.n_uni_z;
    volatile float vol = L[0] * L[1];
    vol = vol * L[2];
    volatile float dens = (float)d.n_atoms / vol;
    volatile float ratio = (float)8 / dens;
    float w = powf(ratio, (float)(1.0 / 3.0));
    if (w > cph) w = cph;
    int n[2], nn[2];
    for (int k = 0; k < 2; k++) {
        n[k] = (int)floorf(L[k] / w);
        if (n[k] < 1) return fail(e, OG_ERR_INVALID, "box too small for one column");
        S.L_cell[k] = L[k] / (float)n[k];
        nn[k] = (int)ceilf(cp / S.L_cell[k]);
        if (nn[k] > n[k])
            return fail(e, OG_ERR_INVALID,
                        "box too small: neighbour reach %d exceeds %d columns (the reference indexes out of range)",
                        nn[k], n[k]);
    }
    S.nx = n[0];
    S.ny = n[1];
    S.n_columns = n[0] * n[1];
    S.n_nb[0] = nn[0];
    S.n_nb[1] = nn[1];
    S.n_nb_cols = (2 * nn[0] + 1) * (2 * nn[1] + 1);
    // ZeroMultipoleSum::set_zms_params, alpha = 0 (float members)
    float c = (float)d.cutoff;
    float c2 = c * c, c3 = c2 * c;
    S.fcoeff = (float)(1.0 / (double)c3);
    S.bcoeff = (float)(0.5 * (double)S.fcoeff);
    S.zcore = erfcf(c * 0.0f) / c + S.bcoeff * c2;
    S.cutoff = (double)c;
    S.cutoff2 = (float)((double)d.cutoff * (double)d.cutoff);
    // An atom that moves farther in one step than the list margin (nsgrid_cutoff - cutoff, at
    // least 1 A) has left every list built for it: the system has blown up.
    const double margin = std::max(d.nsgrid_cutoff - d.cutoff, 1.0);
    S.max_step_disp2 = margin * margin;
    const double half = 0.5 * (d.nsgrid_cutoff - d.cutoff);
    S.list_trig2 = (float)(half * half);
    return OG_OK;
}

// ZeroMultipoleSum::cal_self_energy (ZeroMultipoleSum.cpp:43-106) with its float running sum.
double self_energy(const HostSystem &h) {
    const int n = h.d.n_atoms;
    std::vector<double> dw(n, 0.0);
    for (int k = 0; k < h.n_excess; k++) {
        int i = h.excess[2 * k], j = h.excess[2 * k + 1];
        dw[i] += (double)(float)h.charge[j];
        dw[j] += (double)(float)h.charge[i];
    }
    float mon = 0.0f;
    const double zm = (double)(h.ele.generic ? h.ele.zmcore : h.dev.zcore);
    const float piew = h.ele.generic ? h.ele.piewald : 0.0f;
    for (int i = 0; i < n; i++) {
        double q = (double)(float)h.charge[i];
        double es = ((double)(-piew * (float)q * (float)q) - zm * q * (q + dw[i])) * 0.5 * OG_CHARGE_COEFF;
        mon = (float)((double)mon + es);
    }
    return (double)mon;
}

// ZeroMultipoleSum's constructor and set_zms_params (ZeroMultipoleSum.cpp:6-28,108-202): the
// float coefficients as the reference's float members hold them (float operands, double
// literals), the same formulas in double for the FP64 excluded-pair term, and the self energy's
// core constant of the order (cal_self_energy, ZeroMultipoleSum.cpp:71-77).
void ele_setup(EleDev &E, const og_system_desc &d) {
    E = EleDev{};
    E.mode = d.ele_mode;
    E.hps = d.hps != 0;
    const float c = (float)d.cutoff, a = (float)d.ele_alpha;
    E.alpha = a;
    E.alpha0 = (double)a < 1e-10;
    E.generic = !(E.mode == OG_ELE_ZD && E.alpha0 && !E.hps);
    E.hps_eps = (float)d.hps_epsilon;
    {
        const float c2 = c * c, c3 = c2 * c, c4 = c2 * c2, c5 = c3 * c2, c6 = c3 * c3, c7 = c3 * c4;
        const float tmp = c * a, erc = erfcf(tmp), expterm = expf(-tmp * tmp);
        float f, hz, d1, d2, d3, d4;
        if (E.alpha0) {
            f = (float)(1.0 / c3);
            hz = (float)(2.0 / c3);
            d1 = (float)(1.0 / c2);
            d2 = (float)(2.0 / c3);
            d3 = (float)(6.0 / c4);
            d4 = (float)(24.0 / c5);
        } else {
            const float root_pi = (float)sqrt(3.14159265);  // CelesteObject::PI
            E.piewald = (float)(2.0 / root_pi * a);
            f = erc / c3 + E.piewald * expterm / c2;
            const float t3 = tmp * tmp * tmp, t5 = t3 * tmp * tmp, t7 = t5 * tmp * tmp;
            hz = (float)((erc + expterm * (tmp + t3) * 2.0 / root_pi) * 2.0 / c3);
            d1 = (float)((erc + expterm * tmp * 2.0 / root_pi) / c2);
            d2 = (float)((erc + expterm * (tmp + t3) * 2.0 / root_pi) * 2.0 / c3);
            d3 = (float)((erc + expterm * (tmp + 2.0 / 3.0 * t3 + 2.0 / 3.0 * t5) * 2.0 / root_pi) * 6.0 / c4);
            d4 = (float)((erc + expterm * (tmp + 2.0 / 3.0 * t3 + 1.0 / 6.0 * t5 + 1.0 / 3.0 + t7) * 2.0 / root_pi) *
                         24.0 / c5);
        }
        E.fcoeff = f;
        E.bcoeff = (float)(0.5 * f);
        E.zq2 = (float)(-3.0 / 4.0 * f - hz / 4.0);
        E.zq4 = (float)(f / 8.0 / c2 + hz / 8.0 / c2);
        E.zq22 = (float)(2.0 * E.zq2);
        E.zq44 = (float)(4.0 * E.zq4);
        E.zo2 = (float)(-15.0 / 16.0 * d1 / c - 7.0 / 16.0 * d2 - 1.0 / 16.0 * d3 * c);
        E.zo4 = (float)(5.0 / 16.0 * d1 / c3 + 5.0 / 16.0 * d2 / c2 + 1.0 / 16.0 * d3 / c);
        E.zo6 = (float)(-1.0 / 16.0 * d1 / c5 - 1.0 / 16.0 * d2 / c4 - 1.0 / 48.0 * d3 / c3);
        E.zo22 = (float)(2.0 * E.zo2);
        E.zo44 = (float)(4.0 * E.zo4);
        E.zo66 = (float)(6.0 * E.zo6);
        E.zh2 = (float)(-35.0 / 32.0 * d1 / c - 19.0 / 32.0 * d2 - 1.0 / 96.0 * d4 * c2 - 1.0 / 8.0 * d3 * c);
        E.zh4 = (float)(1.0 / 64.0 * d4 + 35.0 / 64.0 * d1 / c3 + 35.0 / 64.0 * d2 / c2 + 5.0 / 32.0 * d3 / c);
        E.zh6 = (float)(-7.0 / 32.0 * d1 / c5 - 7.0 / 32.0 * d2 / c4 - 1.0 / 12.0 * d3 / c3 - 1.0 / 96.0 * d4 / c2);
        E.zh8 = (float)(5.0 / 128.0 * d2 / c6 + 5.0 / 128.0 * d1 / c7 + 1.0 / 64.0 * d3 / c5 + 1.0 / 384.0 * d4 / c4);
        E.zh22 = (float)(2.0 * E.zh2);
        E.zh44 = (float)(4.0 * E.zh4);
        E.zh66 = (float)(6.0 * E.zh6);
        E.zh88 = (float)(8.0 * E.zh8);
        E.zcore = erc / c + E.bcoeff * c2;
        E.zqcore = erc / c - E.zq2 * c2 - E.zq4 * c4;
        E.zocore = erc / c - E.zo2 * c2 - E.zo4 * c4 - E.zo6 * c6;
        E.zhcore = erc / c - E.zh2 * c2 - E.zh4 * c4 - E.zh6 * c6 - E.zh8 * c6 * c2;
    }
    E.zmcore = E.mode == OG_ELE_ZD ? E.zcore : E.mode == OG_ELE_ZQ ? E.zqcore : E.mode == OG_ELE_ZO ? E.zocore
             : E.mode == OG_ELE_ZH ? E.zhcore : 0.0f;
    if (E.mode == OG_ELE_DH) {
        // CelesteObject.cpp:31-39 constants
        E.dielectric_inv = (float)(1.0 / d.dh_dielectric);
        E.debye_inv = (float)(1.0 / (sqrt(8.85418782e-12 * d.dh_dielectric * 1.380658e-23 * d.dh_temperature /
                                          (2 * 6.0221413e23 * 1.60217657e-19 * 1.60217657e-19 * d.dh_ionic_strength)) *
                                     1e10));
    }
    {  // double precision
        const double c = d.cutoff, a = d.ele_alpha;
        const double c2 = c * c, c3 = c2 * c, c4 = c2 * c2, c5 = c3 * c2, c6 = c3 * c3, c7 = c3 * c4;
        const double tmp = c * a, erc = erfc(tmp), expterm = exp(-tmp * tmp);
        double hz, d1, d2, d3, d4;
        E.d_alpha = a;
        if (E.alpha0) {
            E.d_fcoeff = 1.0 / c3;
            hz = 2.0 / c3;
            d1 = 1.0 / c2;
            d2 = 2.0 / c3;
            d3 = 6.0 / c4;
            d4 = 24.0 / c5;
        } else {
            const double root_pi = sqrt(3.14159265);
            E.d_piewald = 2.0 / root_pi * a;
            E.d_fcoeff = erc / c3 + E.d_piewald * expterm / c2;
            const double t3 = tmp * tmp * tmp, t5 = t3 * tmp * tmp, t7 = t5 * tmp * tmp;
            hz = (erc + expterm * (tmp + t3) * 2.0 / root_pi) * 2.0 / c3;
            d1 = (erc + expterm * tmp * 2.0 / root_pi) / c2;
            d2 = (erc + expterm * (tmp + t3) * 2.0 / root_pi) * 2.0 / c3;
            d3 = (erc + expterm * (tmp + 2.0 / 3.0 * t3 + 2.0 / 3.0 * t5) * 2.0 / root_pi) * 6.0 / c4;
            d4 = (erc + expterm * (tmp + 2.0 / 3.0 * t3 + 1.0 / 6.0 * t5 + 1.0 / 3.0 + t7) * 2.0 / root_pi) * 24.0 / c5;
        }
        const double f = E.d_fcoeff;
        E.d_bcoeff = 0.5 * f;
        E.d_zq2 = -3.0 / 4.0 * f - hz / 4.0;
        E.d_zq4 = f / 8.0 / c2 + hz / 8.0 / c2;
        E.d_zq22 = 2.0 * E.d_zq2;
        E.d_zq44 = 4.0 * E.d_zq4;
        E.d_zo2 = -15.0 / 16.0 * d1 / c - 7.0 / 16.0 * d2 - 1.0 / 16.0 * d3 * c;
        E.d_zo4 = 5.0 / 16.0 * d1 / c3 + 5.0 / 16.0 * d2 / c2 + 1.0 / 16.0 * d3 / c;
        E.d_zo6 = -1.0 / 16.0 * d1 / c5 - 1.0 / 16.0 * d2 / c4 - 1.0 / 48.0 * d3 / c3;
        E.d_zo22 = 2.0 * E.d_zo2;
        E.d_zo44 = 4.0 * E.d_zo4;
        E.d_zo66 = 6.0 * E.d_zo6;
        E.d_zh2 = -35.0 / 32.0 * d1 / c - 19.0 / 32.0 * d2 - 1.0 / 96.0 * d4 * c2 - 1.0 / 8.0 * d3 * c;
        E.d_zh4 = 1.0 / 64.0 * d4 + 35.0 / 64.0 * d1 / c3 + 35.0 / 64.0 * d2 / c2 + 5.0 / 32.0 * d3 / c;
        E.d_zh6 = -7.0 / 32.0 * d1 / c5 - 7.0 / 32.0 * d2 / c4 - 1.0 / 12.0 * d3 / c3 - 1.0 / 96.0 * d4 / c2;
        E.d_zh8 = 5.0 / 128.0 * d2 / c6 + 5.0 / 128.0 * d1 / c7 + 1.0 / 64.0 * d3 / c5 + 1.0 / 384.0 * d4 / c4;
        E.d_zh22 = 2.0 * E.d_zh2;
        E.d_zh44 = 4.0 * E.d_zh4;
        E.d_zh66 = 6.0 * E.d_zh6;
        E.d_zh88 = 8.0 * E.d_zh8;
    }
}

// MmSystem::set_nb15off + set_excess_pairs (MmSystem.cpp:478-525, 700-736): rows in insertion
// order, then pairs i < j walking the rows.
// Exclusion partners per atom as CSR (h.xs, h.xl): each row keeps the order in which the pairs
// list its partners, without repeats, and the excluded ("excess") pairs i < j follow row by row
// (MmSystem::set_excess_pairs, whose order the self energy's float running sum depends on).
og_status build_exclusions(og_engine *e, HostSystem &h) {
    const int n = h.d.n_atoms;
    std::vector<int32_t> deg(n + 1, 0);
    for (int k = 0; k < h.d.n_excl; k++) {
        int a = h.excl[2 * k], b = h.excl[2 * k + 1];
        if (a < 0 || b < 0 || a >= n || b >= n || a == b) return fail(e, OG_ERR_INVALID, "bad exclusion pair %d", k);
        deg[a]++;
        deg[b]++;
    }
    std::vector<int32_t> start(n + 1, 0);
    for (int i = 0; i < n; i++) start[i + 1] = start[i] + deg[i];
    std::vector<int32_t> fill(start.begin(), start.end() - 1), raw(start[n]);
    for (int k = 0; k < h.d.n_excl; k++) {
        int a = h.excl[2 * k], b = h.excl[2 * k + 1];
        raw[fill[a]++] = b;
        raw[fill[b]++] = a;
    }
    h.xs.assign(n + 1, 0);
    h.xl.clear();
    h.xl.reserve(raw.size());
    for (int i = 0; i < n; i++) {
        const size_t row0 = h.xl.size();
        for (int p = start[i]; p < start[i + 1]; p++) {
            bool seen = false;
            for (size_t q = row0; q < h.xl.size(); q++) seen |= h.xl[q] == raw[p];
            if (!seen) h.xl.push_back(raw[p]);
        }
        h.xs[i + 1] = (int32_t)h.xl.size();
    }
    h.excess.clear();
    for (int i = 0; i < n; i++)
        for (int p = h.xs[i]; p < h.xs[i + 1]; p++)
            if (i < h.xl[p]) {
                h.excess.push_back(i);
                h.excess.push_back(h.xl[p]);
            }
    h.n_excess = (int)h.excess.size() / 2;
    return OG_OK;
}

// ---------------------------------------------------------- device scan

template <typename TI>
og_status scan_exclusive(og_engine *e, const TI *in, long long *out, long long n, int level) {
    const long long nb = (n + 2047) / 2048;
    if (level >= (int)e->d_scan_tmp.size() / 2) return fail(e, OG_ERR_CAPACITY, "scan depth");
    long long *sums = e->d_scan_tmp[2 * level], *sums_out = e->d_scan_tmp[2 * level + 1];
    k_scan_block<TI><<<(unsigned)nb, 1024, 0, e->stream>>>(in, out, n, nb > 1 ? sums : nullptr);
    LAUNCH_CHECK();
    if (nb > 1) {
        og_status s = scan_exclusive<long long>(e, sums, sums_out, nb, level + 1);
        if (s) return s;
        k_scan_add<<<blocks(n, 256), 256, 0, e->stream>>>(out, n, sums_out);
        LAUNCH_CHECK();
    }
    return OG_OK;
}

// ---------------------------------------------------------- list build

og_status build_list(og_engine *e) {
    cudaStream_t st = e->stream;
    if (e->d_xq_build) CK(cudaMemsetAsync(e->d_counters + OG_CNT_LIST_STALE, 0, sizeof(int), st));
    CK(cudaMemsetAsync(e->d_col_count, 0, sizeof(int) * e->n_cols, st));
    CK(cudaMemsetAsync(e->d_col_fill, 0, sizeof(int) * e->n_cols, st));
    k_assign_columns<<<blocks(e->n_atoms, 256), 256, 0, st>>>(e->d_sys, e->d_atom_sys, e->d_crd, e->n_atoms,
                                                               e->d_atom_col, e->d_atom_key, e->d_col_count,
                                                               e->d_counters, e->d_sys_fault);
    LAUNCH_CHECK();
    k_scan_columns<<<1, 1024, 0, st>>>(e->d_col_count, e->n_cols, e->d_col_atom_start, e->d_col_cell_start,
                                       e->d_col_head_cell, e->d_counters, e->d_sys_col_base, e->n_sys,
                                       e->d_sys_cell_base);
    LAUNCH_CHECK();
    k_scatter_columns<<<blocks(e->n_atoms, 256), 256, 0, st>>>(e->d_atom_col, e->d_atom_key, e->n_atoms,
                                                                e->d_col_atom_start, e->d_col_fill, e->d_col_keys);
    LAUNCH_CHECK();
    k_sort_columns<<<e->n_cols, 512, 0, st>>>(e->d_col_count, e->d_col_atom_start, e->d_col_cell_start, e->d_col_sys,
                                              e->d_col_keys, e->d_sys, e->d_crd, e->d_slot_atom, e->d_slot_crd,
                                              e->d_atom_slot, e->d_cell_col, e->d_cell_sys, e->d_counters,
                                              e->d_sys_fault);
    LAUNCH_CHECK();
    k_fill_int<<<blocks(e->n_uni, 256), 256, 0, st>>>(e->d_uni_lo, e->n_uni, 0x7fffffff);
    LAUNCH_CHECK();
    k_fill_int<<<blocks(e->n_uni, 256), 256, 0, st>>>(e->d_uni_hi, e->n_uni, -1);
    LAUNCH_CHECK();
    k_cell_info<<<blocks(e->cells_cap, 256), 256, 0, st>>>(e->d_counters, e->cells_cap, e->d_cell_col, e->d_cell_sys,
                                                            e->d_col_cell_start, e->d_sys, e->d_slot_crd,
                                                            e->d_slot_atom, e->d_cell_origin, e->d_cell_zr,
                                                            e->d_cell_uni, e->d_cell_valid, e->d_uni_lo, e->d_uni_hi);
    LAUNCH_CHECK();
    k_slot_refresh<<<blocks(e->slots_cap, 256), 256, 0, st>>>(e->d_counters, e->slots_cap, e->d_slot_atom,
                                                               e->d_slot_crd, e->d_cell_origin, e->d_charge_f,
                                                               e->d_atom_type, e->d_xq, e->d_slot_type);
    LAUNCH_CHECK();
    if (e->d_xq_build)
        CK(cudaMemcpyAsync(e->d_xq_build, e->d_xq, sizeof(float4) * (size_t)e->slots_cap, cudaMemcpyDeviceToDevice, st));
    k_cell_excl<<<blocks(e->cells_cap, 256), 256, 0, st>>>(e->d_counters, e->cells_cap, e->d_slot_atom,
                                                            e->d_atom_slot, e->d_excl_start, e->d_excl_list,
                                                            e->d_cell_excl);
    LAUNCH_CHECK();
    const long long n_items = (long long)e->cells_cap * e->nnc;
    k_count_pairs<<<blocks(n_items, 256), 256, 0, st>>>(e->d_counters, e->cells_cap, e->nnc, e->d_cell_sys,
                                                         e->d_sys_cell_base, e->d_sys, e->d_cell_col,
                                                         e->d_col_cell_start, e->d_col_head_cell, e->d_cell_zr,
                                                         e->d_cell_uni, e->d_uni_lo, e->d_uni_hi, e->d_sys_fault,
                                                         e->d_count);
    LAUNCH_CHECK();
    og_status s = scan_exclusive<int>(e, e->d_count, e->d_offset, n_items + 1, 0);
    if (s) return s;
    k_pair_heads<<<blocks(e->cells_cap + 1, 256), 256, 0, st>>>(e->d_counters, e->cells_cap, e->nnc, e->pair_cap,
                                                                 e->d_offset, e->d_cp_head);
    LAUNCH_CHECK();
    k_fill_pairs<<<blocks(n_items, 256), 256, 0, st>>>(
        e->d_counters, e->cells_cap, e->nnc, e->pair_cap, e->d_cell_sys, e->d_sys_cell_base, e->d_sys, e->d_cell_col,
        e->d_col_cell_start, e->d_col_head_cell, e->d_cell_zr, e->d_cell_uni, e->d_uni_lo, e->d_uni_hi,
        e->d_sys_fault, e->d_offset, e->d_cp_c2img);
    LAUNCH_CHECK();
    k_pair_records<<<blocks((long long)e->cells_cap * 32, 256), 256, 0, st>>>(
        e->d_counters, e->pair_cap, e->d_cell_sys, e->d_sys, e->d_cp_head, e->d_cp_c2img, e->d_cell_valid,
        e->d_slot_atom, e->d_atom_slot, e->d_excl_start, e->d_excl_list, e->d_cell_excl, e->d_cell_origin,
        e->d_cp_mask, e->d_cp_shift);
    LAUNCH_CHECK();
    if (e->d_jl) {  // new list: every system's j lists are rebuilt
        CK(cudaMemsetAsync(e->d_jl_stale, 1, sizeof(int) * e->n_sys, st));
        CK(cudaMemsetAsync(e->d_counters + OG_CNT_JL_STALE, 1, sizeof(int), st));
    }
    return OG_OK;
}

// ---------------------------------------------------------- forces

#define PAIR_ARGS                                                                                            \
    e->d_counters, e->d_cell_sys, e->d_sys, e->d_bbox, e->d_xq, e->d_slot_type, e->d_cp_head, e->d_cp_shift, \
        e->d_cp_c2img, e->d_cp_mask, e->d_lj, e->d_frc, e->d_cell_acc, e->pair_cap
#define JQ_ARGS PAIR_ARGS, e->d_ele, e->d_hps
#define JL_ARGS                                                                                                 \
    e->d_counters, e->d_cell_sys, e->d_sys, e->d_xq, e->d_slot_type, e->d_cp_head, e->d_cp_shift, e->d_cp_c2img, \
        e->d_jl, e->d_jl_count, e->d_lj, e->d_frc, e->d_cell_acc, e->d_ele, e->d_hps, e->d_jl_stale, e->n_sys

// Pair kernel variants differ in the register budget per thread (resident blocks per SM).
// ene = false: the caller does not read this step's energies (only variants 5-6 skip them).
og_status launch_pair(og_engine *e, bool vir, int variant, bool ene) {
    const unsigned nb = blocks((long long)e->cells_cap * 32, 256);
    cudaStream_t st = e->stream;
    // variants 0-2: warp per 8x8 cell pair (register budgets 100/80/64); 3-4: j-major (100/80);
    // 5-6: j-major with packed FP32x2 arithmetic (128/80); 7-9: the same with a j-atom queue
    // (128/80 in blocks of 256, 102 in blocks of 128).  The virial kernel is that of the
    // variant's family.
    // a system with another electrostatics / nonbond model: the generic j-queue (or j-list) kernel
    if (e->any_gen && variant != OG_JL_VARIANT) {
        if (vir) k_pair_ljzd_jq<true, true, 2, 256, true><<<nb, 256, 0, st>>>(JQ_ARGS);
        else if (ene) k_pair_ljzd_jq<false, true, 5, 128, true><<<2 * nb, 128, 0, st>>>(JQ_ARGS);
        else k_pair_ljzd_jq<false, false, 5, 128, true><<<2 * nb, 128, 0, st>>>(JQ_ARGS);
        LAUNCH_CHECK();
        return OG_OK;
    }
    if (variant == OG_PAIR_VARIANT_F64) {
        if (!e->d_lj64) return fail(e, OG_ERR_STATE, "FP64 pair variant without its FP64 LJ table");
        if (vir)
            k_pair_f64<true><<<nb, 256, 0, st>>>(e->d_counters, e->d_cell_sys, e->d_sys, e->d_slot_crd, e->d_slot_atom,
                                                 e->d_slot_type, e->d_charge, e->d_cp_head, e->d_cp_c2img,
                                                 e->d_cp_mask, e->d_lj64, e->pair_cap, e->d_frc, e->d_cell_acc);
        else
            k_pair_f64<false><<<nb, 256, 0, st>>>(e->d_counters, e->d_cell_sys, e->d_sys, e->d_slot_crd,
                                                  e->d_slot_atom, e->d_slot_type, e->d_charge, e->d_cp_head,
                                                  e->d_cp_c2img, e->d_cp_mask, e->d_lj64, e->pair_cap, e->d_frc,
                                                  e->d_cell_acc);
        LAUNCH_CHECK();
        return OG_OK;
    }
    if (variant == OG_JL_VARIANT) {
        if (!e->d_jl) return fail(e, OG_ERR_STATE, "pair variant %d without its j lists", OG_JL_VARIANT);
        k_jl_build<256><<<nb, 256, 0, st>>>(e->d_counters, e->d_cell_sys, e->d_sys, e->d_bbox, e->d_xq,
                                                 e->d_cp_head, e->d_cp_shift, e->d_cp_mask, e->pair_cap,
                                                 2.0f * e->jl_skin + 1e-3f, e->d_jl, e->d_jl_count, e->d_xq_ref,
                                                 e->d_jl_stale);
        LAUNCH_CHECK();
        if (e->any_gen) {
            if (vir) k_pair_ljzd_jl<true, true, 2, 128, true><<<2 * nb, 128, 0, st>>>(JL_ARGS);
            else if (ene) k_pair_ljzd_jl<false, true, 5, 128, true><<<2 * nb, 128, 0, st>>>(JL_ARGS);
            else k_pair_ljzd_jl<false, false, 5, 128, true><<<2 * nb, 128, 0, st>>>(JL_ARGS);
        } else if (vir) {
            k_pair_ljzd_jl<true, true, 2, 128, false><<<2 * nb, 128, 0, st>>>(JL_ARGS);
        } else if (ene) {
            k_pair_ljzd_jl<false, true, 5, 128, false><<<2 * nb, 128, 0, st>>>(JL_ARGS);
        } else {
            k_pair_ljzd_jl<false, false, 5, 128, false><<<2 * nb, 128, 0, st>>>(JL_ARGS);
        }
        LAUNCH_CHECK();
        return OG_OK;
    }
    if (vir && variant >= 7) k_pair_ljzd_jq<true, true, 2, 256, false><<<nb, 256, 0, st>>>(JQ_ARGS);
    else if (vir && variant >= 5) k_pair_ljzd_jm2<true, true, 2><<<nb, 256, 0, st>>>(PAIR_ARGS);
    else if (vir && variant >= 3) k_pair_ljzd_jm<true, 2><<<nb, 256, 0, st>>>(PAIR_ARGS);
    else if (vir) k_pair_ljzd<true, 2><<<nb, 256, 0, st>>>(PAIR_ARGS);
    else if (variant == 1) k_pair_ljzd<false, 3><<<nb, 256, 0, st>>>(PAIR_ARGS);
    else if (variant == 2) k_pair_ljzd<false, 4><<<nb, 256, 0, st>>>(PAIR_ARGS);
    else if (variant == 3) k_pair_ljzd_jm<false, 2><<<nb, 256, 0, st>>>(PAIR_ARGS);
    else if (variant == 4) k_pair_ljzd_jm<false, 3><<<nb, 256, 0, st>>>(PAIR_ARGS);
    else if (variant == 5 && ene) k_pair_ljzd_jm2<false, true, 2><<<nb, 256, 0, st>>>(PAIR_ARGS);
    else if (variant == 5) k_pair_ljzd_jm2<false, false, 2><<<nb, 256, 0, st>>>(PAIR_ARGS);
    else if (variant == 6 && ene) k_pair_ljzd_jm2<false, true, 3><<<nb, 256, 0, st>>>(PAIR_ARGS);
    else if (variant == 6) k_pair_ljzd_jm2<false, false, 3><<<nb, 256, 0, st>>>(PAIR_ARGS);
    else if (variant == 7 && ene) k_pair_ljzd_jq<false, true, 2, 256, false><<<nb, 256, 0, st>>>(JQ_ARGS);
    else if (variant == 7) k_pair_ljzd_jq<false, false, 2, 256, false><<<nb, 256, 0, st>>>(JQ_ARGS);
    else if (variant == 8 && ene) k_pair_ljzd_jq<false, true, 3, 256, false><<<nb, 256, 0, st>>>(JQ_ARGS);
    else if (variant == 8) k_pair_ljzd_jq<false, false, 3, 256, false><<<nb, 256, 0, st>>>(JQ_ARGS);
    else if (variant == 9 && ene) k_pair_ljzd_jq<false, true, 5, 128, false><<<2 * nb, 128, 0, st>>>(JQ_ARGS);
    else if (variant == 9) k_pair_ljzd_jq<false, false, 5, 128, false><<<2 * nb, 128, 0, st>>>(JQ_ARGS);
    else k_pair_ljzd<false, 2><<<nb, 256, 0, st>>>(PAIR_ARGS);
    LAUNCH_CHECK();
    return OG_OK;
}

og_status reduce_potential(og_engine *e);
og_status reduce_virial(og_engine *e);

// ene = false: this step's energies are not read (see run_step); forces are the same.
og_status compute_forces(og_engine *e, bool vir, bool ene = true) {
    cudaStream_t st = e->stream;
    const unsigned pair_blocks = blocks((long long)e->cells_cap * 32, 256);
    k_cell_bbox<<<blocks(e->cells_cap, 256), 256, 0, st>>>(e->d_counters, e->cells_cap, e->d_xq, e->d_cell_valid,
                                                            e->d_bbox);
    LAUNCH_CHECK();
    if (e->timing == 1) {
        if (e->pev_used >= (int)e->pev0.size()) {
            cudaEvent_t a, b;
            CK(cudaEventCreate(&a));
            CK(cudaEventCreate(&b));
            e->pev0.push_back(a);
            e->pev1.push_back(b);
        }
        CK(cudaEventRecord(e->pev0[e->pev_used], st));
    }
    {
        og_status ps = launch_pair(e, vir, e->pair_variant, ene || vir);
        if (ps) return ps;
    }
    if (e->timing == 1) CK(cudaEventRecord(e->pev1[e->pev_used++], st));
    if (vir) {
        if (!e->d_vir_atom) {
            og_status s = dalloc(e, &e->d_vir_atom, 9 * (size_t)e->n_atoms);
            if (s) return s;
            s = dalloc(e, &e->d_vir_exc, 9 * (size_t)(e->n_excess + 1));
            if (s) return s;
        }
        k_atom_virial<<<blocks(e->n_atoms, 256), 256, 0, st>>>(e->n_atoms, e->d_atom_slot, e->d_frc, e->d_xq,
                                                                e->d_cell_origin, e->d_vir_atom);
        LAUNCH_CHECK();
    }
    if (e->n_excess) {
        k_excess<<<blocks(e->n_excess, 256), 256, 0, st>>>(e->n_excess, e->d_excess, e->d_excess_sys, e->d_sys,
                                                            e->d_ele, e->d_crd, e->d_charge, e->d_atom_slot, e->d_frc,
                                                            e->d_e_exc, vir ? e->d_vir_exc : nullptr);
        LAUNCH_CHECK();
    }
    if (e->n_bonds) {
        k_bonds<<<blocks(e->n_bonds, 256), 256, 0, st>>>(e->n_bonds, e->d_bond, e->d_bond_kr, e->d_bond_sys, e->d_sys,
                                                          e->d_crd, e->d_atom_slot, e->d_frc, e->d_e_bond);
        LAUNCH_CHECK();
    }
    if (e->n_angles) {
        k_angles<<<blocks(e->n_angles, 256), 256, 0, st>>>(e->n_angles, e->d_angle, e->d_angle_kt, e->d_sys,
                                                            e->d_crd, e->d_atom_slot, e->d_frc, e->d_e_angle);
        LAUNCH_CHECK();
    }
    if (e->n_tors) {
        k_dihedrals<<<blocks(e->n_tors, 128), 128, 0, st>>>(e->n_tors, e->d_tors, e->d_tors_p, e->d_tors_sys, e->d_sys,
                                                             e->d_crd, e->d_atom_slot, e->d_frc, e->d_e_tors);
        LAUNCH_CHECK();
    }
    if (e->n_impro) {
        k_dihedrals<<<blocks(e->n_impro, 128), 128, 0, st>>>(e->n_impro, e->d_impro, e->d_impro_p, e->d_impro_sys,
                                                              e->d_sys, e->d_crd, e->d_atom_slot, e->d_frc,
                                                              e->d_e_impro);
        LAUNCH_CHECK();
    }
    if (e->n_nb14) {
        k_nb14<<<blocks(e->n_nb14, 128), 128, 0, st>>>(e->n_nb14, e->d_nb14, e->d_nb14_t, e->d_nb14_c, e->d_nb14_sys,
                                                        e->d_sys, e->d_crd, e->d_charge_f, e->d_lj, e->d_atom_slot,
                                                        e->d_frc, e->d_e_nb14);
        LAUNCH_CHECK();
    }
    k_collect_slots<<<blocks(e->slots_cap, 256), 256, 0, st>>>(e->d_counters, e->slots_cap, e->d_slot_atom, e->d_frc,
                                                                e->d_work);
    LAUNCH_CHECK();
    og_status rs = OG_OK;
    if ((ene || vir) && (rs = reduce_potential(e))) return rs;
    if (vir && (rs = reduce_virial(e))) return rs;
    return OG_OK;
}

// Two-level fixed-order sum of NV fields over every system's segment into out[s*stride + off].
template <int NV>
og_status seg_sum(og_engine *e, const double *v, int vstride, int field0, const int *base, int max_chunks,
                  double *out, int out_stride, int out_off, int accumulate) {
    dim3 grid(max_chunks, e->n_sys);
    k_part<NV><<<grid, 256, 0, e->stream>>>(v, vstride, field0, base, max_chunks, e->d_part);
    LAUNCH_CHECK();
    k_part_final<NV><<<e->n_sys, 256, 0, e->stream>>>(e->d_part, max_chunks, out, out_stride, out_off, nullptr,
                                                      accumulate);
    LAUNCH_CHECK();
    return OG_OK;
}

og_status reduce_potential(og_engine *e) {
    og_status s;
    if ((s = seg_sum<2>(e, e->d_cell_acc, OG_CELL_ACC, 0, e->d_sys_cell_base, e->mc_cells, e->d_sys_acc, OG_ACC_SIZE,
                        OG_ACC_VDW, 0)))
        return s;
    if (e->n_excess && (s = seg_sum<1>(e, e->d_e_exc, 1, 0, e->d_seg_exc, e->mc_exc, e->d_sys_acc, OG_ACC_SIZE,
                                       OG_ACC_EXCESS, 0)))
        return s;
    if (e->n_bonds && (s = seg_sum<1>(e, e->d_e_bond, 1, 0, e->d_seg_bond, e->mc_bond, e->d_sys_acc, OG_ACC_SIZE,
                                      OG_ACC_BOND, 0)))
        return s;
    if (e->n_angles && (s = seg_sum<1>(e, e->d_e_angle, 1, 0, e->d_seg_angle, e->mc_angle, e->d_sys_acc,
                                       OG_ACC_SIZE, OG_ACC_ANGLE, 0)))
        return s;
    if (e->n_tors && (s = seg_sum<1>(e, e->d_e_tors, 1, 0, e->d_seg_tors, e->mc_tors, e->d_sys_acc, OG_ACC_SIZE,
                                     OG_ACC_TORSION, 0)))
        return s;
    if (e->n_impro && (s = seg_sum<1>(e, e->d_e_impro, 1, 0, e->d_seg_impro, e->mc_impro, e->d_sys_acc,
                                      OG_ACC_SIZE, OG_ACC_IMPRO, 0)))
        return s;
    if (e->n_nb14 && (s = seg_sum<2>(e, e->d_e_nb14, 2, 0, e->d_seg_nb14, e->mc_nb14, e->d_sys_acc, OG_ACC_SIZE,
                                     OG_ACC_VDW14, 0)))
        return s;
    k_vmcmd<<<e->n_sys, 32, 0, e->stream>>>(e->n_sys, e->d_sys, e->d_vstates, e->d_sys_acc, e->d_step, e->vm_advance,
                                             e->d_vs_cur, e->d_mt, e->d_vs_log, e->d_lambda_log, e->vm_log_cap,
                                             e->d_mcmd);
    LAUNCH_CHECK();
    return OG_OK;
}

og_status reduce_virial(og_engine *e) {
    og_status s;
    if ((s = seg_sum<10>(e, e->d_cell_acc, OG_CELL_ACC, 2, e->d_sys_cell_base, e->mc_cells, e->d_sys_acc,
                         OG_ACC_SIZE, OG_ACC_VIR, 0)))
        return s;
    if ((s = seg_sum<9>(e, e->d_vir_atom, 9, 0, e->d_seg_atoms, e->mc_atoms, e->d_sys_acc, OG_ACC_SIZE, OG_ACC_VIR,
                        1)))
        return s;
    if (e->n_excess && (s = seg_sum<9>(e, e->d_vir_exc, 9, 0, e->d_seg_exc, e->mc_exc, e->d_sys_acc, OG_ACC_SIZE,
                                       OG_ACC_VIR, 1)))
        return s;
    return OG_OK;
}

og_status com_cancel(og_engine *e, double *v, const int *active) {
    if (!e->any_groups) return OG_OK;
    dim3 grid(e->mc_grp, e->n_groups);
    k_part_momentum<<<grid, 256, 0, e->stream>>>(e->d_grp_start, e->d_grp_atoms, e->d_mass, v, e->d_grp_sys, active,
                                                 e->mc_grp, e->d_part);
    LAUNCH_CHECK();
    k_part_final<3><<<e->n_groups, 256, 0, e->stream>>>(e->d_part, e->mc_grp, e->d_moment, 3, 0, e->d_grp_mass_inv, 0);
    LAUNCH_CHECK();
    k_com_apply<<<blocks(e->n_atoms, 256), 256, 0, e->stream>>>(e->n_atoms, e->d_atom_group, e->d_moment,
                                                                 e->d_atom_sys, active, v);
    LAUNCH_CHECK();
    return OG_OK;
}

og_status shake(og_engine *e, const int *active) {
    cudaStream_t st = e->stream;
    if (e->n_spair) {
        k_shake_pair<<<blocks(e->n_spair, 128), 128, 0, st>>>(e->n_spair, e->d_spair, e->d_spair_d2, e->d_spair_sys,
                                                               e->d_sys, active, e->d_mass_inv, e->d_crd,
                                                               e->d_crd_prev);
        LAUNCH_CHECK();
    }
    if (e->n_strio) {
        k_shake_trio<<<blocks(e->n_strio, 128), 128, 0, st>>>(e->n_strio, e->d_strio, e->d_strio_d2, e->d_sys,
                                                               active, e->d_mass_inv, e->d_crd, e->d_crd_prev,
                                                               e->shake_max_loops, e->shake_tol, e->d_counters);
        LAUNCH_CHECK();
    }
    if (e->n_squad) {
        k_shake_quad<<<blocks(e->n_squad, 64), 64, 0, st>>>(e->n_squad, e->d_squad, e->d_squad_d2, e->d_squad_sys,
                                                             e->d_sys, active, e->d_mass_inv, e->d_crd, e->d_crd_prev,
                                                             e->shake_max_loops, e->shake_tol, e->d_counters);
        LAUNCH_CHECK();
    }
    return OG_OK;
}

// One pass of ThermostatScaling::apply_thermostat_with_shake's loop (Thermostat.cpp:105-170) for
// the systems still in d_active: constraint, temperature test, rescale, COM cancel, positions.
// In a graph, the pass in which every system leaves the loop still launches the later kernels;
// they skip inactive systems, so the state is the one the reference's `break` leaves.
og_status thermo_pass(og_engine *e, cudaGraphConditionalHandle cond, int use_cond) {
    cudaStream_t st = e->stream;
    og_status s = shake(e, e->d_active);
    if (s) return s;
    k_ke_mid<<<blocks(e->n_atoms, 256), 256, 0, st>>>(e->n_atoms, e->d_mass, e->d_vel, e->d_vel_next, e->d_ke);
    LAUNCH_CHECK();
    if ((s = seg_sum<1>(e, e->d_ke, 1, 0, e->d_seg_atoms, e->mc_atoms, e->d_sum_tmp, 1, 0, 0))) return s;
    k_thermo_check<<<blocks(e->n_sys, 128), 128, 0, st>>>(e->n_sys, e->d_sys, e->d_sum_tmp, e->d_thermo, e->d_step,
                                                           e->d_thermo_it, e->thermo_max_loops, e->thermo_tol,
                                                           e->d_active, e->d_any, e->d_counters);
    LAUNCH_CHECK();
    if (!use_cond) CK(cudaMemcpyAsync(e->h_pinned, e->d_any, sizeof(int), cudaMemcpyDeviceToHost, st));
    k_thermo_next<<<1, 32, 0, st>>>(e->d_any, e->d_thermo_it, e->thermo_max_loops, cond, use_cond);
    LAUNCH_CHECK();
    if (!use_cond) {
        CK(cudaStreamSynchronize(st));
        if (e->h_pinned[0] == 0) return OG_OK;
    }
    k_thermo_half<<<blocks(e->n_atoms, 256), 256, 0, st>>>(e->n_atoms, e->d_atom_sys, e->d_sys, e->d_active,
                                                            e->d_work, e->d_mass, e->d_mass_inv, e->d_crd,
                                                            e->d_buf_crd, e->d_vel, e->d_vel_next, e->d_ke);
    LAUNCH_CHECK();
    if ((s = seg_sum<1>(e, e->d_ke, 1, 0, e->d_seg_atoms, e->mc_atoms, e->d_sum_tmp, 1, 0, 0))) return s;
    k_thermo_rescale<<<blocks(e->n_atoms, 256), 256, 0, st>>>(e->n_atoms, e->d_atom_sys, e->d_sys, e->d_active,
                                                               e->d_sum_tmp, e->d_thermo, e->d_step, e->d_work,
                                                               e->d_mass_inv, e->d_crd, e->d_buf_crd, e->d_vel,
                                                               e->d_vel_next);
    LAUNCH_CHECK();
    s = com_cancel(e, e->d_vel_next, e->d_active);
    if (s) return s;
    k_thermo_crd<<<blocks(e->n_atoms, 256), 256, 0, st>>>(e->n_atoms, e->d_atom_sys, e->d_sys, e->d_active, e->d_crd,
                                                           e->d_crd_prev, e->d_vel_next);
    LAUNCH_CHECK();
    return OG_OK;
}

// ThermostatScaling::apply_thermostat_with_shake (Thermostat.cpp:86-170) for every system that
// has constraints and the scaling thermostat; the loop ends when all have converged or after
// thermo_const_max_loops passes.  Launched directly, the host reads the "still iterating"
// count after every pass.  Under graph capture the loop becomes a conditional WHILE node whose
// body is one pass; k_thermo_next sets its condition on the device.
og_status thermostat_with_shake(og_engine *e) {
    cudaStream_t st = e->stream;
    if (e->thermo_max_loops <= 0) return OG_OK;
    CK(cudaMemcpyAsync(e->d_active, e->d_mask_thermo, sizeof(int) * e->n_sys, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemsetAsync(e->d_any, 0, sizeof(int), st));
    CK(cudaMemsetAsync(e->d_thermo_it, 0, sizeof(int), st));
    k_copy_double<<<blocks(3LL * e->n_atoms, 256), 256, 0, st>>>(e->d_buf_crd, e->d_crd, 3LL * e->n_atoms);
    LAUNCH_CHECK();
    if (!e->capturing) {
        for (int it = 0; it < e->thermo_max_loops; it++) {
            og_status s = thermo_pass(e, cudaGraphConditionalHandle(), 0);
            if (s) return s;
            if (e->h_pinned[0] == 0) break;
        }
        return OG_OK;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t n_deps = 0;
    CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &n_deps));
    if (cs != cudaStreamCaptureStatusActive || !g) return fail(e, OG_ERR_STATE, "thermostat loop: stream not capturing");
    cudaGraphConditionalHandle cond;
    CK(cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = cond;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, n_deps, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    CK(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    CK(cudaStreamBeginCaptureToGraph(e->side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    e->stream = e->side;
    og_status s = thermo_pass(e, cond, 1);
    e->stream = st;
    cudaGraph_t captured = nullptr;
    cudaError_t r = cudaStreamEndCapture(e->side, &captured);
    if (s) return s;
    CK(r);
    return OG_OK;
}

// Displacement list policy, kernel by kernel: the host reads the counters (one copy and a stream
// synchronisation per step) and builds the list when it is stale and no system has faulted in
// this call (as k_list_cond decides inside a graph).
og_status build_list_if_stale(og_engine *e) {
    CK(cudaMemcpyAsync(e->h_pinned + 8, e->d_counters, sizeof(int) * OG_CNT_SIZE, cudaMemcpyDeviceToHost,
                       e->stream));
    CK(cudaStreamSynchronize(e->stream));
    const int *c = e->h_pinned + 8;
    const bool fault = (c[OG_CNT_FLAGS] & (OG_FLAG_BAD_COORD | OG_FLAG_COLUMN_CAPACITY | OG_FLAG_DISPLACEMENT)) != 0;
    if (!c[OG_CNT_LIST_STALE] || fault) return OG_OK;
    e->host_cond_builds++;
    return build_list(e);
}

// Displacement list policy inside a captured graph: a conditional IF node whose body is the list
// build, its condition set on the device from the stale mark (k_list_cond), so replays rebuild
// exactly when an atom has moved half the margin.
og_status build_list_if_stale_captured(og_engine *e) {
    cudaStream_t st = e->stream;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t n_deps = 0;
    CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &n_deps));
    if (cs != cudaStreamCaptureStatusActive || !g) return fail(e, OG_ERR_STATE, "list build: stream not capturing");
    cudaGraphConditionalHandle cond;
    CK(cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault));
    k_list_cond<<<1, 32, 0, st>>>(e->d_counters, cond);
    LAUNCH_CHECK();
    CK(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &n_deps));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = cond;
    np.conditional.type = cudaGraphCondTypeIf;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, n_deps, &np));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    CK(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    CK(cudaStreamBeginCaptureToGraph(e->side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    e->stream = e->side;
    const long long l0 = e->launches;
    og_status s = build_list(e);
    e->cond_build_kernels = e->launches - l0;  // counted per build that runs, not per replay
    e->launches = l0;
    e->stream = st;
    cudaGraph_t captured = nullptr;
    cudaError_t r = cudaStreamEndCapture(e->side, &captured);
    if (s) return s;
    CK(r);
    return OG_OK;
}

// ene: evaluate this step's energies.  They are needed on every step when a system is
// McMD-scaled (the factor depends on the potential) or the energy trace is on, and otherwise
// only on the last step of a call, whose energies og_get_energies reads.
og_status run_step(og_engine *e, bool ene) {
    cudaStream_t st = e->stream;
    og_status s;
    if (e->list_policy == OG_LIST_DISPLACEMENT) {
        s = e->capturing ? build_list_if_stale_captured(e) : build_list_if_stale(e);
        if (s) return s;
    } else if (e->host_step % e->intvl == 0) {
        s = build_list(e);
        if (s) return s;
    }
    e->vm_advance = 1;  // V-McMD transitions and logs belong to steps only
    s = compute_forces(e, false, ene || e->any_mcmd || e->trace_cap > 0);
    e->vm_advance = 0;
    if (s) return s;
    k_update_velocities<<<blocks(e->n_atoms, 256), 256, 0, st>>>(e->n_atoms, e->d_atom_sys, e->d_sys, e->d_mcmd,
                                                                  e->d_work, e->d_mass_inv, e->d_vel,
                                                                  e->d_vel_next);
    LAUNCH_CHECK();
    s = com_cancel(e, e->d_vel_next, nullptr);
    if (s) return s;
    if (e->any_thermo_free) {
        k_thermo_scaling_ke<<<blocks(e->n_atoms, 256), 256, 0, st>>>(e->n_atoms, e->d_atom_sys, e->d_sys, e->d_work,
                                                                      e->d_mass, e->d_mass_inv, e->d_vel, e->d_ke);
        LAUNCH_CHECK();
        if ((s = seg_sum<1>(e, e->d_ke, 1, 0, e->d_seg_atoms, e->mc_atoms, e->d_sum_tmp, 1, 0, 0))) return s;
        k_thermo_scaling_apply<<<blocks(e->n_atoms, 256), 256, 0, st>>>(e->n_atoms, e->d_atom_sys, e->d_sys,
                                                                         e->d_sum_tmp, e->d_thermo, e->d_step,
                                                                         e->d_work, e->d_mass_inv, e->d_vel,
                                                                         e->d_vel_next);
        LAUNCH_CHECK();
    }
    k_update_coordinates<<<blocks(e->n_atoms, 256), 256, 0, st>>>(e->n_atoms, e->d_atom_sys, e->d_sys, e->d_crd,
                                                                   e->d_crd_prev, e->d_vel_next);
    LAUNCH_CHECK();
    if (e->any_plain_cons) {
        s = shake(e, e->d_mask_plain);
        if (s) return s;
    }
    if (e->any_thermo_cons) {
        s = thermostat_with_shake(e);
        if (s) return s;
    }
    k_finish<<<blocks(e->n_atoms, 256), 256, 0, st>>>(e->n_atoms, e->d_atom_sys, e->d_sys, 1, e->d_crd,
                                                       e->d_crd_prev, e->d_vel, e->d_vel_next, e->d_atom_slot,
                                                       e->d_slot_crd, e->d_cell_origin, e->d_xq, e->d_mass, e->d_ke,
                                                       e->d_counters, e->d_sys_fault, e->d_xq_ref,
                                                       e->jl_skin * e->jl_skin, e->d_jl_stale, e->d_xq_build);
    LAUNCH_CHECK();
    if ((s = seg_sum<1>(e, e->d_ke, 1, 0, e->d_seg_atoms, e->mc_atoms, e->d_sys_acc, OG_ACC_SIZE, OG_ACC_KIN, 0)))
        return s;
    k_energies<<<blocks(e->n_sys, 128), 128, 0, st>>>(e->n_sys, e->d_sys, e->d_sys_acc, e->d_mcmd, e->d_energies,
                                                       e->d_trace, e->trace_cap, e->d_trace_count);
    LAUNCH_CHECK();
    if (e->n_tr_entries) {
        k_capture_frames<<<blocks(e->n_tr_entries, 256), 256, 0, st>>>(e->n_tr_entries, e->d_tr_atom, e->d_tr_sys,
                                                                        e->d_tr_idx, e->d_sys, e->d_step,
                                                                        e->d_crd_prev, e->d_energies, e->d_frames,
                                                                        e->d_frame_ene);
        LAUNCH_CHECK();
    }
    k_trace_advance<<<1, 32, 0, st>>>(e->d_trace_count, e->d_step);
    LAUNCH_CHECK();
    e->host_step++;
    return OG_OK;
}

// ---- V-McMD logs: the device rings hold the entries of recent steps; these move them to the
// host before a ring would wrap.
long long vm_entries_end(long long g, int intvl) {  // entries of steps 0..g-1: k = 1..result
    return g > 0 ? (g - 1) / intvl : 0;
}

void logs_update_limit(og_engine *e) {
    long long lim = LLONG_MAX;
    for (int m = 0; m < e->n_vm; m++) {
        const SysDev &D = e->sys[e->vm_sys[m]].dev;
        const VmLog &L = e->vm[m];
        lim = std::min(lim, (L.vs_next_k + e->vm_log_cap) * D.vs_trans_intvl - D.first_step);
        if (D.vs_lambda_intvl > 0)
            lim = std::min(lim, (L.lam_next_k + e->vm_log_cap) * D.vs_lambda_intvl - D.first_step);
    }
    // frame k is written at the end of step k * interval - 1
    for (int m = 0; m < e->n_tr; m++) {
        const SysDev &D = e->sys[e->tr_sys[m]].dev;
        lim = std::min(lim, (e->tr[m].next_k + D.tr_frames) * D.tr_interval - 1 - D.first_step);
    }
    e->log_limit = lim;
}

// Moves the trajectory frames of the steps run so far to the host (the stream is synchronised).
og_status frames_drain(og_engine *e) {
    for (int m = 0; m < e->n_tr; m++) {
        const SysDev &D = e->sys[e->tr_sys[m]].dev;
        TrLog &T = e->tr[m];
        const long long ke = (D.first_step + e->host_step) / D.tr_interval;  // frames of steps < g
        const size_t fc = 3 * (size_t)D.tr_n;
        for (long long k = T.next_k; k <= ke; k++) {
            const long long slot = (k - 1) % D.tr_frames;
            const size_t c0 = T.crd.size(), e0 = T.ene.size();
            T.crd.resize(c0 + fc);
            T.ene.resize(e0 + OG_N_ENERGY);
            CK(cudaMemcpyAsync(T.crd.data() + c0, e->d_frames + D.tr_crd_base + slot * fc, sizeof(float) * fc,
                               cudaMemcpyDeviceToHost, e->stream));
            CK(cudaMemcpyAsync(T.ene.data() + e0, e->d_frame_ene + D.tr_ene_base + slot * OG_N_ENERGY,
                               sizeof(double) * OG_N_ENERGY, cudaMemcpyDeviceToHost, e->stream));
            T.step.push_back(k * D.tr_interval);
            T.next_k = k + 1;
        }
    }
    CK(cudaStreamSynchronize(e->stream));
    return OG_OK;
}

// Synchronises the stream and moves every ring entry of the steps run so far to the host.
og_status logs_drain(og_engine *e) {
    if (e->n_tr) {
        og_status s = frames_drain(e);
        if (s) return s;
    }
    if (e->n_vm == 0) {
        logs_update_limit(e);
        return OG_OK;
    }
    const size_t n = (size_t)e->n_vm * e->vm_log_cap;
    std::vector<int32_t> vs(n);
    std::vector<double> lam(n);
    CK(cudaMemcpyAsync(vs.data(), e->d_vs_log, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, e->stream));
    CK(cudaMemcpyAsync(lam.data(), e->d_lambda_log, sizeof(double) * n, cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    for (int m = 0; m < e->n_vm; m++) {
        const SysDev &D = e->sys[e->vm_sys[m]].dev;
        VmLog &L = e->vm[m];
        const long long g = D.first_step + e->host_step;
        const size_t ring = (size_t)m * e->vm_log_cap;
        for (long long k = L.vs_next_k, ke = vm_entries_end(g, D.vs_trans_intvl); k <= ke; k++) {
            L.vs_step.push_back(k * D.vs_trans_intvl);
            L.vs.push_back(vs[ring + (size_t)((k - 1) % e->vm_log_cap)]);
            L.vs_next_k = k + 1;
        }
        if (D.vs_lambda_intvl > 0)
            for (long long k = L.lam_next_k, ke = vm_entries_end(g, D.vs_lambda_intvl); k <= ke; k++) {
                L.lam_step.push_back(k * D.vs_lambda_intvl);
                L.lam.push_back(lam[ring + (size_t)((k - 1) % e->vm_log_cap)]);
                L.lam_next_k = k + 1;
            }
    }
    logs_update_limit(e);
    return OG_OK;
}

// Before steps [host_step, host_step + n): drain first when a ring would wrap during them.
og_status logs_reserve(og_engine *e, long long n) {
    if ((e->n_vm == 0 && e->n_tr == 0) || e->host_step + n <= e->log_limit) return OG_OK;
    return logs_drain(e);
}

template <class T>
og_status vm_take(og_engine *e, int32_t sys, int64_t max, int64_t *step, T *val, int64_t *n, bool vs_log) {
    if (!e || !e->finalized) return fail(e, OG_ERR_STATE, "V-McMD log read before og_finalize");
    if (sys < 0 || sys >= e->n_sys || max < 0 || !n || (max > 0 && (!step || !val)))
        return fail(e, OG_ERR_INVALID, "bad system id or output arrays");
    const int m = e->sys[sys].dev.vm_slot;
    if (m < 0) return fail(e, OG_ERR_INVALID, "system %d has no V-McMD transitions", sys);
    og_status s = logs_drain(e);
    if (s) return s;
    VmLog &L = e->vm[m];
    std::vector<long long> &st = vs_log ? L.vs_step : L.lam_step;
    std::vector<T> &v = *reinterpret_cast<std::vector<T> *>(vs_log ? (void *)&L.vs : (void *)&L.lam);
    size_t &head = vs_log ? L.vs_head : L.lam_head;
    const int64_t avail = (int64_t)(st.size() - head);
    if (max == 0) {
        *n = avail;
        return OG_OK;
    }
    const int64_t k = std::min(max, avail);
    for (int64_t i = 0; i < k; i++) {
        step[i] = st[head + i];
        val[i] = v[head + i];
    }
    head += (size_t)k;
    if (head == st.size()) {
        st.clear();
        v.clear();
        head = 0;
    }
    *n = k;
    return OG_OK;
}

og_status read_counters(og_engine *e, int *out) {
    CK(cudaMemcpyAsync(e->h_pinned, e->d_counters, sizeof(int) * OG_CNT_SIZE, cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    memcpy(out, e->h_pinned, sizeof(int) * OG_CNT_SIZE);
    e->builds_seen = out[OG_CNT_LIST_BUILDS];
    return OG_OK;
}

og_status check_flags(og_engine *e) {
    int c[OG_CNT_SIZE];
    og_status s = read_counters(e, c);
    if (s) return s;
    int f = c[OG_CNT_FLAGS];
    if (f & OG_FLAG_BAD_COORD) return fail(e, OG_ERR_INVALID, "non-finite or far out-of-box coordinate");
    if (f & OG_FLAG_COLUMN_CAPACITY)
        return fail(e, OG_ERR_CAPACITY, "a MiniCell column holds more than %d atoms", OG_MAX_COLUMN_ATOMS);
    if (f & OG_FLAG_PAIR_CAPACITY)
        return fail(e, OG_ERR_CAPACITY, "cell-pair list needs %d entries, capacity %lld", c[OG_CNT_N_PAIRS], e->pair_cap);
    return OG_OK;
}

void drop_graph(og_engine *e) {
    if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
    e->graph_exec = nullptr;
    if (e->graph1_exec) cudaGraphExecDestroy(e->graph1_exec);
    e->graph1_exec = nullptr;
}

og_status grow_pairs(og_engine *e, long long need) {
    drop_graph(e);  // the graph holds the old list buffers
    long long cap = need + need / 2 + 4096;
    dfree(e, e->d_cp_c2img);
    dfree(e, e->d_cp_mask);
    dfree(e, e->d_cp_shift);
    e->d_cp_c2img = nullptr;
    e->d_cp_mask = nullptr;
    e->d_cp_shift = nullptr;
    og_status s = dalloc(e, &e->d_cp_c2img, (size_t)cap);
    if (s) return s;
    s = dalloc(e, &e->d_cp_mask, (size_t)cap);
    if (s) return s;
    s = dalloc(e, &e->d_cp_shift, (size_t)cap);
    if (s) return s;
    e->pair_cap = cap;
    if (e->d_jl) {
        dfree(e, e->d_jl);
        e->d_jl = nullptr;
        s = dalloc(e, &e->d_jl, 8 * (size_t)cap);
        if (s) return s;
    }
    return OG_OK;
}

// The j lists of the pair variant OG_JL_VARIANT (8 entries per cell-pair record), their counts and
// the positions they are built from; marked stale, so the first pair launch builds them.
og_status jl_alloc(og_engine *e) {
    if (e->d_jl) return OG_OK;
    if ((long long)e->slots_cap >= (1ll << 24))
        return fail(e, OG_ERR_INVALID, "pair variant %d needs fewer than 2^24 atom slots (engine has %d)",
                    OG_JL_VARIANT, e->slots_cap);
    const char *env = getenv("OG_JL_SKIN");
    if (env && *env) e->jl_skin = std::min(2.0f, std::max(0.05f, (float)atof(env)));
    og_status s;
    if ((s = dalloc(e, &e->d_jl, 8 * (size_t)e->pair_cap)) || (s = dalloc(e, &e->d_jl_count, (size_t)e->cells_cap)) ||
        (s = dalloc(e, &e->d_xq_ref, (size_t)e->slots_cap)) || (s = dalloc(e, &e->d_jl_stale, (size_t)e->n_sys)))
        return s;
    CK(cudaMemsetAsync(e->d_jl_stale, 1, sizeof(int) * e->n_sys, e->stream));
    CK(cudaMemsetAsync(e->d_counters + OG_CNT_JL_STALE, 1, sizeof(int), e->stream));
    return OG_OK;
}

void jl_free(og_engine *e) {
    dfree(e, e->d_jl);
    dfree(e, e->d_jl_count);
    dfree(e, e->d_xq_ref);
    dfree(e, e->d_jl_stale);
    e->d_jl = nullptr;
    e->d_jl_count = nullptr;
    e->d_xq_ref = nullptr;
    e->d_jl_stale = nullptr;
}

// Captures one list interval -- the rebuild step and the intvl-1 steps after it -- into a graph.
// Kernel arguments are device pointers and sizes fixed at og_finalize; the step number, the
// thermostat loop index and every per-step decision live on the device, so the graph replays
// any interval.  A failed capture turns graphs off for the engine (kernel-by-kernel steps give
// the same results) and records why.
og_status capture_interval(og_engine *e) {
    const long long step0 = e->host_step, launches0 = e->launches;
    CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeRelaxed));
    e->capturing = true;
    og_status s = OG_OK;
    for (int i = 0; i < e->intvl && s == OG_OK; i++) s = run_step(e, i == e->intvl - 1);
    e->capturing = false;
    cudaGraph_t g = nullptr;
    cudaError_t r = cudaStreamEndCapture(e->stream, &g);
    e->host_step = step0;
    e->graph_kernels = e->launches - launches0;
    e->launches = launches0;
    if (s == OG_OK && r == cudaSuccess && g) r = cudaGraphInstantiate(&e->graph_exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (s != OG_OK || r != cudaSuccess || !e->graph_exec) {
        cudaGetLastError();
        e->graph_exec = nullptr;
        e->use_graphs = false;
        e->graph_note = s != OG_OK ? e->err : std::string(cudaGetErrorString(r));
    }
    return OG_OK;
}

// One step with energies as a graph (og_step_async's single steps under the displacement
// policy).  A failed capture leaves single steps kernel by kernel; the interval graphs of
// og_step are not affected.
og_status capture_one_step(og_engine *e) {
    const long long step0 = e->host_step, launches0 = e->launches;
    CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeRelaxed));
    e->capturing = true;
    og_status s = run_step(e, true);
    e->capturing = false;
    cudaGraph_t g = nullptr;
    cudaError_t r = cudaStreamEndCapture(e->stream, &g);
    e->host_step = step0;
    e->graph1_kernels = e->launches - launches0;
    e->launches = launches0;
    if (s == OG_OK && r == cudaSuccess && g) r = cudaGraphInstantiate(&e->graph1_exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (s != OG_OK || r != cudaSuccess || !e->graph1_exec) {
        cudaGetLastError();
        e->graph1_exec = nullptr;
        e->graph1_failed = true;
    }
    return OG_OK;
}

og_status clear_flags(og_engine *e) {
    CK(cudaMemsetAsync(e->d_counters + OG_CNT_FLAGS, 0, sizeof(int), e->stream));
    CK(cudaMemsetAsync(e->d_sys_fault, 0, sizeof(int) * e->n_sys, e->stream));
    return OG_OK;
}

// Builds the list and grows the pair buffer until it fits (synchronous; used at setup and
// after a capacity miss).
og_status build_list_checked(og_engine *e) {
    for (int attempt = 0; attempt < 4; attempt++) {
        og_status s = clear_flags(e);
        if (s) return s;
        s = build_list(e);
        if (s) return s;
        int c[OG_CNT_SIZE];
        s = read_counters(e, c);
        if (s) return s;
        if (c[OG_CNT_FLAGS] & OG_FLAG_PAIR_CAPACITY) {
            s = grow_pairs(e, c[OG_CNT_N_PAIRS]);
            if (s) return s;
            continue;
        }
        return check_flags(e);
    }
    return fail(e, OG_ERR_CAPACITY, "cell-pair list did not fit after growing");
}

// Times each pair-kernel variant on the first list (3 launches each, best of three) and keeps
// the fastest; OG_PAIR_VARIANT=0/1/2 in the environment fixes the choice.  The trial launches
// write the force accumulators, which are cleared afterwards.
og_status autotune_pair(og_engine *e) {
    // the other electrostatics / nonbond models have generic instantiations of variants 9 and 10
    // only; a fixed choice of another variant falls back to 9
    const char *env = getenv("OG_PAIR_VARIANT");
    if (e->fixed_variant == OG_PAIR_VARIANT_F64) {
        if (e->any_gen)
            return fail(e, OG_ERR_INVALID, "the FP64 pair variant evaluates zero-dipole alpha = 0 with plain LJ only");
        e->pair_variant = OG_PAIR_VARIANT_F64;
        return OG_OK;
    }
    if (e->fixed_variant >= 0 || (env && *env)) {
        e->pair_variant = e->fixed_variant >= 0 ? e->fixed_variant : atoi(env) % OG_N_PAIR_VARIANTS;
        if (e->any_gen && e->pair_variant != OG_JL_VARIANT) e->pair_variant = 9;
        return e->pair_variant == OG_JL_VARIANT ? jl_alloc(e) : OG_OK;
    }
    k_cell_bbox<<<blocks(e->cells_cap, 256), 256, 0, e->stream>>>(e->d_counters, e->cells_cap, e->d_xq,
                                                                   e->d_cell_valid, e->d_bbox);
    LAUNCH_CHECK();
    const bool try_jl = (long long)e->slots_cap < (1ll << 24);
    if (try_jl) {
        og_status s = jl_alloc(e);
        if (s) return s;
    }
    double best = 1e30;
    for (int v = 0; v < OG_N_PAIR_VARIANTS; v++) {
        if ((v == OG_JL_VARIANT && !try_jl) || (e->any_gen && v != 9 && v != OG_JL_VARIANT)) {
            e->variant_ms[v] = 0.0;
            continue;
        }
        double vbest = 1e30, first = 0.0;
        for (int rep = 0; rep < 3; rep++) {
            CK(cudaEventRecord(e->ev_pair0, e->stream));
            og_status s = launch_pair(e, false, v, false);
            if (s) return s;
            CK(cudaEventRecord(e->ev_pair1, e->stream));
            CK(cudaEventSynchronize(e->ev_pair1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e->ev_pair0, e->ev_pair1));
            if (v == OG_JL_VARIANT && rep == 0) first = ms;  // the j lists are built once, here
            else vbest = std::min(vbest, (double)ms);
        }
        // the j lists are rebuilt at every cell-pair list build and whenever an atom passes the
        // skin: on water at 2 fs about once per 2.4 steps (42 builds per 100 steps at 1M atoms, 8 in
        // 20 at the start of a run), so the build is charged at one per two steps, not one per
        // list interval
        if (v == OG_JL_VARIANT) vbest += std::max(0.0, first - vbest) * OG_JL_BUILDS_PER_STEP;
        e->variant_ms[v] = vbest;
        if (vbest < best) {
            best = vbest;
            e->pair_variant = v;
        }
    }
    // Near-ties go to the j-list kernel.  Each variant sums its FP32 pair terms in its own order,
    // so a choice that a timing within a few percent decides would change a trajectory's last
    // bits from one run to the next (the 87k-atom chain times variants 9 and 10 within 0.3%).
    if (try_jl && e->variant_ms[OG_JL_VARIANT] <= 1.05 * best) e->pair_variant = OG_JL_VARIANT;
    if (try_jl && e->pair_variant != OG_JL_VARIANT) jl_free(e);
    CK(cudaMemsetAsync(e->d_frc, 0, sizeof(unsigned long long) * 3 * (size_t)e->slots_cap, e->stream));
    return OG_OK;
}

}  // namespace

// ======================================================================= C ABI

extern "C" {

og_status og_create(int device, og_engine **out) {
    if (!out) return OG_ERR_INVALID;
    *out = nullptr;
    og_engine *e = new og_engine();
    e->device = device;
    const char *poison = getenv("OG_DEBUG_POISON");
    if (poison && *poison) e->poison = atoi(poison) & 0xff;
    cudaError_t r = cudaSetDevice(device);
    if (r != cudaSuccess) {
        delete e;
        return OG_ERR_CUDA;
    }
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&e->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&e->ev_pair0) != cudaSuccess || cudaEventCreate(&e->ev_pair1) != cudaSuccess ||
        cudaEventCreate(&e->ev_step0) != cudaSuccess || cudaEventCreate(&e->ev_step1) != cudaSuccess ||
        cudaMallocHost((void **)&e->h_pinned, 64 * sizeof(int)) != cudaSuccess) {
        delete e;
        return OG_ERR_CUDA;
    }
    *out = e;
    return OG_OK;
}

og_status og_destroy(og_engine *e) {
    if (!e) return OG_OK;
    cudaSetDevice(e->device);
    if (e->stream) {
        cudaStreamSynchronize(e->stream);
        for (void *p : e->allocs) cudaFreeAsync(p, e->stream);
        cudaStreamSynchronize(e->stream);
    }
    e->allocs.clear();
    if (e->h_pinned) cudaFreeHost(e->h_pinned);
    for (auto ev : e->pev0) cudaEventDestroy(ev);
    for (auto ev : e->pev1) cudaEventDestroy(ev);
    if (e->ev_pair0) cudaEventDestroy(e->ev_pair0);
    if (e->ev_pair1) cudaEventDestroy(e->ev_pair1);
    if (e->ev_step0) cudaEventDestroy(e->ev_step0);
    if (e->ev_step1) cudaEventDestroy(e->ev_step1);
    if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
    if (e->graph1_exec) cudaGraphExecDestroy(e->graph1_exec);
    if (e->stream) cudaStreamDestroy(e->stream);
    if (e->side) cudaStreamDestroy(e->side);
    delete e;
    return OG_OK;
}

const char *og_last_error(const og_engine *e) { return e ? e->err.c_str() : "null engine"; }

og_status og_add_system(og_engine *e, const og_system_desc *d, int32_t *sys_id) {
    if (!e || !d) return OG_ERR_INVALID;
    if (e->finalized) return fail(e, OG_ERR_STATE, "og_add_system after og_finalize");
    const int n = d->n_atoms;
    if (n <= 0 || !d->crd || !d->vel || !d->charge || !d->mass || !d->atom_type || d->n_lj_types <= 0 || !d->lj6 ||
        !d->lj12)
        return fail(e, OG_ERR_INVALID, "system needs atoms, coordinates, velocities, charges, masses and LJ tables");
    if (d->cutoff <= 0 || d->nsgrid_cutoff < d->cutoff || d->time_step <= 0 || d->nsgrid_update_intvl <= 0)
        return fail(e, OG_ERR_INVALID, "need 0 < cutoff <= nsgrid_cutoff, time_step > 0, nsgrid_update_intvl > 0");
    if (!e->sys.empty() && d->nsgrid_update_intvl != e->intvl)
        return fail(e, OG_ERR_INVALID, "all systems of one engine share nsgrid_update_intvl");
    if (d->mcmd_order > 7) return fail(e, OG_ERR_INVALID, "McMD polynomial order above 7");
    if (d->n_vstates < 0 || (d->n_vstates > 0 && (!d->vs_order || !d->vs_lambda || !d->vs_prob || !d->vs_coef ||
                                                   d->vmcmd_trans_interval < 1 || d->vmcmd_init_vs < 0 ||
                                                   d->vmcmd_init_vs >= d->n_vstates ||
                                                   d->vmcmd_lambda_log_interval < 0)))
        return fail(e, OG_ERR_INVALID, "V-McMD needs state arrays, trans_interval >= 1 and an initial state in range");
    for (int v = 0; v < d->n_vstates; v++)
        if (d->vs_order[v] < 0 || d->vs_order[v] > 7)
            return fail(e, OG_ERR_INVALID, "virtual state %d: polynomial order outside 0..7", v);
    if (d->n_vstates > 0 && d->vmcmd_mt_state && d->vmcmd_mt_state[624] > 624)
        return fail(e, OG_ERR_INVALID, "V-McMD generator position above 624");
    if (d->ele_mode < OG_ELE_ZD || d->ele_mode > OG_ELE_DH || !(d->ele_alpha >= 0.0) ||
        (d->ele_mode == OG_ELE_DH &&
         !(d->dh_dielectric > 0.0 && d->dh_ionic_strength > 0.0 && d->dh_temperature > 0.0)) ||
        (d->hps && (!d->lj_hps_cutoff || !d->lj_hps_lambda)))
        return fail(e, OG_ERR_INVALID, "electrostatics model: mode 0..4, alpha >= 0, positive Debye-Hueckel "
                    "parameters, HPS tables when hps is on");
    if (d->first_step < 0 || d->first_step % d->nsgrid_update_intvl != 0)
        return fail(e, OG_ERR_INVALID, "first_step must be a non-negative multiple of nsgrid_update_intvl");
    e->sys.emplace_back();
    HostSystem &h = e->sys.back();
    h.d = *d;
    auto cp = [](auto &vec, const auto *src, size_t cnt) {
        vec.assign(src ? src : nullptr, src ? src + cnt : nullptr);
    };
    cp(h.crd, d->crd, 3 * (size_t)n);
    cp(h.vel, d->vel, 3 * (size_t)n);
    cp(h.charge, d->charge, n);
    cp(h.mass, d->mass, n);
    cp(h.type, d->atom_type, n);
    cp(h.lj6, d->lj6, (size_t)d->n_lj_types * d->n_lj_types);
    cp(h.lj12, d->lj12, (size_t)d->n_lj_types * d->n_lj_types);
    cp(h.excl, d->excl, 2 * (size_t)d->n_excl);
    cp(h.sp, d->shake_pair, 2 * (size_t)d->n_shake_pair);
    cp(h.spd, d->shake_pair_dist, d->n_shake_pair);
    cp(h.st, d->shake_trio, 3 * (size_t)d->n_shake_trio);
    cp(h.std_, d->shake_trio_dist, 3 * (size_t)d->n_shake_trio);
    cp(h.bond, d->bond, 2 * (size_t)d->n_bonds);
    cp(h.bk, d->bond_k, d->n_bonds);
    cp(h.br0, d->bond_r0, d->n_bonds);
    cp(h.angle, d->angle, 3 * (size_t)d->n_angles);
    cp(h.ak, d->angle_k, d->n_angles);
    cp(h.at0, d->angle_t0, d->n_angles);
    cp(h.gstart, d->com_group_start, d->n_com_groups > 0 ? d->n_com_groups + 1 : 0);
    if (d->n_com_groups > 0) cp(h.gatoms, d->com_group_atoms, d->com_group_start[d->n_com_groups]);
    if (d->mcmd_order >= 0) cp(h.mcoef, d->mcmd_coef, d->mcmd_order + 1);
    if (d->hps) {
        cp(h.hcut, d->lj_hps_cutoff, (size_t)d->n_lj_types * d->n_lj_types);
        cp(h.hlam, d->lj_hps_lambda, (size_t)d->n_lj_types * d->n_lj_types);
    }
    ele_setup(h.ele, *d);
    if (d->n_vstates > 0) {
        // ExtendedVMcMD::set_vs_params / set_vs_poly_param (Extend.cpp:266-283)
        int c0 = 0;
        for (int v = 0; v < d->n_vstates; v++) {
            VsDev V{};
            V.lo = d->vs_lambda[2 * v];
            V.hi = d->vs_lambda[2 * v + 1];
            V.p_down = d->vs_prob[2 * v];
            V.p_up = d->vs_prob[2 * v + 1];
            V.order = d->vs_order[v];
            for (int i = 0; i <= V.order; i++) V.coef[i] = d->vs_coef[c0 + i];
            c0 += V.order + 1;
            h.vstates.push_back(V);
        }
        h.mt.resize(OG_MT_WORDS);
        if (d->vmcmd_mt_state) {
            std::copy(d->vmcmd_mt_state, d->vmcmd_mt_state + OG_MT_WORDS, h.mt.begin());
        } else {
            // std::mt19937::seed: x0 = seed, x_i = 1812433253 (x_{i-1} ^ (x_{i-1} >> 30)) + i
            h.mt[0] = d->vmcmd_seed;
            for (uint32_t i = 1; i < 624; i++) h.mt[i] = 1812433253u * (h.mt[i - 1] ^ (h.mt[i - 1] >> 30)) + i;
            h.mt[624] = 624;
        }
    } else if (d->mcmd_order >= 0) {
        VsDev V{};
        V.lo = d->mcmd_lambda_low;
        V.hi = d->mcmd_lambda_high;
        V.order = d->mcmd_order;
        for (int i = 0; i <= V.order; i++) V.coef[i] = h.mcoef[i];
        h.vstates.push_back(V);
    }
    if ((d->n_torsions > 0 && (!d->torsion || !d->torsion_ene || !d->torsion_phase || !d->torsion_overlaps ||
                               !d->torsion_symmetry)) ||
        (d->n_impros > 0 && (!d->impro || !d->impro_ene || !d->impro_phase || !d->impro_overlaps ||
                             !d->impro_symmetry)) ||
        (d->n_nb14 > 0 && (!d->nb14 || !d->nb14_type || !d->nb14_coeff_vdw || !d->nb14_coeff_ele)) ||
        (d->n_shake_quad > 0 && (!d->shake_quad || !d->shake_quad_dist)) || d->n_torsions < 0 || d->n_impros < 0 ||
        d->n_nb14 < 0 || d->n_shake_quad < 0 || d->dof_extra < 0) {
        e->sys.pop_back();
        return fail(e, OG_ERR_INVALID, "dihedral, 1-4 or SHAKE-quad arrays missing or negative counts");
    }
    cp(h.tq, d->torsion, 4 * (size_t)d->n_torsions);
    cp(h.tene, d->torsion_ene, d->n_torsions);
    cp(h.tph, d->torsion_phase, d->n_torsions);
    cp(h.tov, d->torsion_overlaps, d->n_torsions);
    cp(h.tsym, d->torsion_symmetry, d->n_torsions);
    cp(h.iq, d->impro, 4 * (size_t)d->n_impros);
    cp(h.iene, d->impro_ene, d->n_impros);
    cp(h.iph, d->impro_phase, d->n_impros);
    cp(h.iov, d->impro_overlaps, d->n_impros);
    cp(h.isym, d->impro_symmetry, d->n_impros);
    cp(h.p14, d->nb14, 2 * (size_t)d->n_nb14);
    cp(h.t14, d->nb14_type, 2 * (size_t)d->n_nb14);
    cp(h.cv14, d->nb14_coeff_vdw, d->n_nb14);
    cp(h.ce14, d->nb14_coeff_ele, d->n_nb14);
    cp(h.qa, d->shake_quad, 4 * (size_t)d->n_shake_quad);
    cp(h.qd, d->shake_quad_dist, 6 * (size_t)d->n_shake_quad);
    {
        auto bad_atoms = [n](const std::vector<int32_t> &v) {
            for (int32_t a : v)
                if (a < 0 || a >= n) return true;
            return false;
        };
        bool bad = bad_atoms(h.tq) || bad_atoms(h.iq) || bad_atoms(h.p14) || bad_atoms(h.qa);
        for (int32_t t : h.t14) bad |= t < 0 || t >= d->n_lj_types;
        for (int32_t o : h.tov) bad |= o == 0;
        for (int32_t o : h.iov) bad |= o == 0;
        for (double q : h.qd) bad |= !(q > 0);
        if (bad) {
            e->sys.pop_back();
            return fail(e, OG_ERR_INVALID, "dihedral, 1-4 or SHAKE-quad entry out of range");
        }
    }
    for (int i = 0; i < n; i++)
        if (h.type[i] < 0 || h.type[i] >= d->n_lj_types || !(h.mass[i] > 0)) {
            e->sys.pop_back();
            return fail(e, OG_ERR_INVALID, "atom %d: bad type or mass", i);
        }
    og_status s = setup_geometry(e, h);
    if (s) {
        e->sys.pop_back();
        return s;
    }
    // MmSystem::revise_crd_inbox (MmSystem.cpp:808-816): wrap into [lower, upper) with the
    // float box bounds
    for (int i = 0; i < n; i++)
        for (int q = 0; q < 3; q++) {
            double &x = h.crd[3 * i + q];
            const double lo = (double)h.dev.lowerf[q], up = (double)h.dev.upperf[q], L = (double)h.dev.Lf[q];
            if (!std::isfinite(x) || std::fabs(x - lo) > 1e4 * L) {
                e->sys.pop_back();
                return fail(e, OG_ERR_INVALID, "atom %d: coordinate not finite or far outside the box", i);
            }
            while (x < lo) x += L;
            while (x >= up) x -= L;
        }
    s = build_exclusions(e, h);
    if (s) {
        e->sys.pop_back();
        return s;
    }
    e->intvl = d->nsgrid_update_intvl;
    if (sys_id) *sys_id = (int32_t)e->sys.size() - 1;
    return OG_OK;
}

og_status og_finalize(og_engine *e) {
    if (!e) return OG_ERR_INVALID;
    if (e->finalized) return fail(e, OG_ERR_STATE, "already finalized");
    if (e->sys.empty()) return fail(e, OG_ERR_STATE, "no systems");
    CK(cudaSetDevice(e->device));
    og_status s;
    const int S = (int)e->sys.size();
    e->n_sys = S;
    // ---- global layout
    std::vector<SysDev> sd(S);
    std::vector<int> atom_sys, col_sys, sys_col_base(S + 1), atom_type, atom_group, excl_start(1, 0), excl_list;
    std::vector<double> crd, vel, charge;
    std::vector<float> charge_f, mass, mass_inv;
    std::vector<float2> lj, hps_tab;
    std::vector<double2> lj64;  // only for the FP64 validation variant
    std::vector<EleDev> ele_tab;
    std::vector<int2> excess, bondv, spair;
    std::vector<int> excess_sys, bond_sys, spair_sys, grp_start(1, 0), grp_atoms, grp_sys;
    std::vector<double2> bond_kr, angle_kt;
    std::vector<int4> anglev, strio;
    std::vector<double> spair_d2, strio_d2, thermo;
    std::vector<float> grp_mass_inv;
    std::vector<int> mask_plain(S), mask_thermo(S);
    std::vector<int4> torsv, improv, squadv;
    std::vector<double4> tors_p, impro_p;
    std::vector<int> tors_sys, impro_sys, nb14_sys, squad_sys;
    std::vector<int2> nb14v, nb14t;
    std::vector<double2> nb14c;
    std::vector<double> squad_d2;
    std::vector<VsDev> vstates;
    std::vector<int> vs_cur;
    std::vector<uint32_t> mt_all;
    std::vector<int> tr_atom, tr_sysv, tr_idx;
    long long tr_crd_total = 0, tr_ene_total = 0;
    {
        size_t n_all = 0, x_all = 0, e_all = 0;
        for (const HostSystem &h : e->sys) {
            n_all += h.d.n_atoms;
            x_all += h.xl.size();
            e_all += h.n_excess;
        }
        for (auto *v : {&atom_sys, &atom_type, &atom_group}) v->reserve(n_all);
        for (auto *v : {&crd, &vel}) v->reserve(3 * n_all);
        charge.reserve(n_all);
        for (auto *v : {&charge_f, &mass, &mass_inv}) v->reserve(n_all);
        excl_start.reserve(n_all + 1);
        excl_list.reserve(x_all);
        excess.reserve(e_all);
        excess_sys.reserve(e_all);
    }
    int atom_base = 0, col_base = 0, uni_base = 0, lj_base = 0, cells_cap = 0, nnc = 1;
    for (int k = 0; k < S; k++) {
        HostSystem &h = e->sys[k];
        SysDev &D = h.dev;
        const og_system_desc &d = h.d;
        const int n = d.n_atoms;
        D.atom_base = atom_base;
        D.n_atoms = n;
        D.col_base = col_base;
        D.uni_base = uni_base;
        D.lj_base = lj_base;
        D.n_types = d.n_lj_types;
        D.dt = d.time_step;
        D.thermostat = d.thermostat;
        D.has_constraints = (d.n_shake_pair + d.n_shake_trio + d.n_shake_quad) > 0;
        h.d_free = 3 * n - 3 - (d.n_shake_pair + 3 * d.n_shake_trio + 6 * d.n_shake_quad) + d.dof_extra;
        if (h.d_free <= 0) return fail(e, OG_ERR_INVALID, "system %d has no degrees of freedom", k);
        D.temperature_coeff_thermo =
            (2.0 * OG_JOULE_CAL * 1e+3) / (OG_GAS_CONST * (double)h.d_free) * OG_KINETIC_COEFF;
        D.temperature_coeff_dyn = 1.0 / (OG_GAS_CONST * (double)h.d_free) * OG_JOULE_CAL * 1e3 * 2.0;
        double tau = d.berendsen_tau;
        if (d.time_step < tau) tau = d.time_step;
        D.tau_inv = 1.0 / tau;
        D.n_vs = (int)h.vstates.size();
        e->any_mcmd |= D.n_vs > 0;
        D.vs_base = (int)vstates.size();
        vstates.insert(vstates.end(), h.vstates.begin(), h.vstates.end());
        D.mcmd_k = (OG_GAS_CONST / OG_JOULE_CAL) * 1e-3 * d.mcmd_temperature;
        D.first_step = d.first_step;
        D.tr_slot = -1;
        D.tr_interval = D.tr_n = D.tr_frames = 0;
        D.tr_crd_base = D.tr_ene_base = 0;
        if (h.tr_interval > 0) {
            // a ring of frames long enough for the frames of one list interval
            D.tr_slot = (int)e->tr_sys.size();
            D.tr_interval = h.tr_interval;
            D.tr_n = (int)h.tr_group.size();
            D.tr_frames = e->intvl / h.tr_interval + 2;
            D.tr_crd_base = tr_crd_total;
            D.tr_ene_base = tr_ene_total;
            tr_crd_total += (long long)D.tr_frames * D.tr_n * 3;
            tr_ene_total += (long long)D.tr_frames * OG_N_ENERGY;
            for (int j = 0; j < D.tr_n; j++) {
                tr_atom.push_back(atom_base + h.tr_group[j]);
                tr_sysv.push_back(k);
                tr_idx.push_back(j);
            }
            e->tr_sys.push_back(k);
        }
        D.vm_slot = -1;
        D.vs_trans_intvl = D.vs_lambda_intvl = 0;
        vs_cur.push_back(d.n_vstates > 0 ? d.vmcmd_init_vs : 0);
        if (d.n_vstates > 0) {
            D.vm_slot = (int)e->vm_sys.size();
            D.vs_trans_intvl = d.vmcmd_trans_interval;
            D.vs_lambda_intvl = d.vmcmd_lambda_log_interval;
            e->vm_sys.push_back(k);
            mt_all.insert(mt_all.end(), h.mt.begin(), h.mt.end());
        }
        D.self_energy = self_energy(h);
        D.excess_base = (int)excess.size();
        D.n_excess = h.n_excess;
        D.bond_base = (int)bondv.size();
        D.n_bonds = d.n_bonds;
        D.angle_base = (int)anglev.size();
        D.n_angles = d.n_angles;
        D.trio_base = (int)strio.size();
        D.n_trio = d.n_shake_trio;
        D.pair_base = (int)spair.size();
        D.n_pair = d.n_shake_pair;
        D.tors_base = (int)torsv.size();
        D.n_tors = d.n_torsions;
        D.impro_base = (int)improv.size();
        D.n_impro = d.n_impros;
        D.nb14_base = (int)nb14v.size();
        D.n_nb14 = d.n_nb14;
        for (int q = 0; q < d.n_torsions; q++) {
            torsv.push_back(make_int4(atom_base + h.tq[4 * q], atom_base + h.tq[4 * q + 1], atom_base + h.tq[4 * q + 2],
                                      atom_base + h.tq[4 * q + 3]));
            tors_p.push_back(make_double4(h.tene[q], h.tph[q], (double)h.tov[q], (double)h.tsym[q]));
            tors_sys.push_back(k);
        }
        for (int q = 0; q < d.n_impros; q++) {
            improv.push_back(make_int4(atom_base + h.iq[4 * q], atom_base + h.iq[4 * q + 1], atom_base + h.iq[4 * q + 2],
                                       atom_base + h.iq[4 * q + 3]));
            impro_p.push_back(make_double4(h.iene[q], h.iph[q], (double)h.iov[q], (double)h.isym[q]));
            impro_sys.push_back(k);
        }
        for (int q = 0; q < d.n_nb14; q++) {
            nb14v.push_back(make_int2(atom_base + h.p14[2 * q], atom_base + h.p14[2 * q + 1]));
            nb14t.push_back(make_int2(h.t14[2 * q], h.t14[2 * q + 1]));
            nb14c.push_back(make_double2(h.cv14[q], h.ce14[q]));
            nb14_sys.push_back(k);
        }
        for (int q = 0; q < d.n_shake_quad; q++) {
            squadv.push_back(make_int4(atom_base + h.qa[4 * q], atom_base + h.qa[4 * q + 1], atom_base + h.qa[4 * q + 2],
                                       atom_base + h.qa[4 * q + 3]));
            for (int r = 0; r < 6; r++) squad_d2.push_back(h.qd[6 * q + r] * h.qd[6 * q + r]);
            squad_sys.push_back(k);
        }
        thermo.push_back(d.temperature);
        thermo.push_back(d.temperature_init < 0 ? d.temperature : d.temperature_init);
        thermo.push_back((double)d.heating_steps);
        thermo.push_back((double)d.first_step);
        mask_plain[k] = D.has_constraints && d.thermostat != OG_THERMOSTAT_SCALING;
        mask_thermo[k] = D.has_constraints && d.thermostat == OG_THERMOSTAT_SCALING;
        e->any_plain_cons |= mask_plain[k] != 0;
        e->any_thermo_cons |= mask_thermo[k] != 0;
        e->any_thermo_free |= (!D.has_constraints && d.thermostat == OG_THERMOSTAT_SCALING);
        if (d.n_shake_trio || d.n_shake_pair || d.n_shake_quad) {
            e->shake_max_loops = d.const_max_loops > 0 ? d.const_max_loops : 1000;
            e->shake_tol = d.const_tolerance > 0 ? d.const_tolerance : 1e-7;
        }
        if (d.thermostat == OG_THERMOSTAT_SCALING) {
            e->thermo_max_loops = d.thermo_const_max_loops > 0 ? d.thermo_const_max_loops : 100;
            e->thermo_tol = d.thermo_const_tolerance > 0 ? d.thermo_const_tolerance : 1e-5;
        }
        for (int i = 0; i < n; i++) {
            atom_sys.push_back(k);
            for (int q = 0; q < 3; q++) {
                crd.push_back(h.crd[3 * i + q]);
                vel.push_back(h.vel[3 * i + q]);
            }
            charge.push_back(h.charge[i]);
            charge_f.push_back((float)h.charge[i]);
            mass.push_back((float)h.mass[i]);
            mass_inv.push_back((float)(1.0 / (double)(float)h.mass[i]));
            atom_type.push_back(h.type[i]);
        }
        // exclusion CSR (global ids), built by og_add_system
        for (int i = 0; i < n; i++) {
            for (int p = h.xs[i]; p < h.xs[i + 1]; p++) excl_list.push_back(atom_base + h.xl[p]);
            excl_start.push_back((int)excl_list.size());
        }
        for (int q = 0; q < (e->pair_only ? 0 : h.n_excess); q++) {
            excess.push_back(make_int2(atom_base + h.excess[2 * q], atom_base + h.excess[2 * q + 1]));
            excess_sys.push_back(k);
        }
        for (int q = 0; q < d.n_bonds; q++) {
            bondv.push_back(make_int2(atom_base + h.bond[2 * q], atom_base + h.bond[2 * q + 1]));
            bond_sys.push_back(k);
            bond_kr.push_back(make_double2(h.bk[q], h.br0[q]));
        }
        for (int q = 0; q < d.n_angles; q++) {
            anglev.push_back(make_int4(atom_base + h.angle[3 * q], atom_base + h.angle[3 * q + 1],
                                       atom_base + h.angle[3 * q + 2], k));
            angle_kt.push_back(make_double2(h.ak[q], h.at0[q]));
        }
        for (int q = 0; q < d.n_shake_pair; q++) {
            spair.push_back(make_int2(atom_base + h.sp[2 * q], atom_base + h.sp[2 * q + 1]));
            spair_sys.push_back(k);
            spair_d2.push_back(h.spd[q] * h.spd[q]);
        }
        for (int q = 0; q < d.n_shake_trio; q++) {
            strio.push_back(make_int4(atom_base + h.st[3 * q], atom_base + h.st[3 * q + 1], atom_base + h.st[3 * q + 2], k));
            for (int r = 0; r < 3; r++) strio_d2.push_back(h.std_[3 * q + r] * h.std_[3 * q + r]);
        }
        // COM groups: MmSystem::set_atom_group_info mass sums in float (MmSystem.cpp:568-584)
        std::vector<int> grp_of(n, -1);
        for (int g = 0; g < d.n_com_groups; g++) {
            float msum = 0.0f;
            for (int q = h.gstart[g]; q < h.gstart[g + 1]; q++) {
                int a = h.gatoms[q];
                if (a < 0 || a >= n) return fail(e, OG_ERR_INVALID, "COM group atom out of range");
                if (grp_of[a] >= 0) return fail(e, OG_ERR_INVALID, "COM groups must be disjoint");
                grp_of[a] = (int)grp_mass_inv.size();
                grp_atoms.push_back(atom_base + a);
                msum += (float)h.mass[a];
            }
            grp_start.push_back((int)grp_atoms.size());
            grp_mass_inv.push_back((float)(1.0 / (double)msum));
            grp_sys.push_back(k);
        }
        for (int i = 0; i < n; i++) atom_group.push_back(grp_of[i]);
        for (int i = 0; i < d.n_lj_types; i++)
            for (int j = 0; j < d.n_lj_types; j++)
                lj.push_back(make_float2((float)h.lj6[i * d.n_lj_types + j], (float)h.lj12[i * d.n_lj_types + j]));
        if (e->fixed_variant == OG_PAIR_VARIANT_F64)
            for (int i = 0; i < d.n_lj_types * d.n_lj_types; i++) lj64.push_back(make_double2(h.lj6[i], h.lj12[i]));
        for (int i = 0; i < d.n_lj_types; i++)
            for (int j = 0; j < d.n_lj_types; j++)
                hps_tab.push_back(h.ele.hps ? make_float2((float)h.hcut[i * d.n_lj_types + j],
                                                          (float)h.hlam[i * d.n_lj_types + j])
                                            : make_float2(0.f, 1.f));
        ele_tab.push_back(h.ele);
        e->any_gen |= h.ele.generic != 0;
        for (int c = 0; c < D.n_columns; c++) col_sys.push_back(k);
        sys_col_base[k] = col_base;
        cells_cap += n / OG_CELL + D.n_columns + 1;
        nnc = std::max(nnc, D.n_nb_cols);
        atom_base += n;
        col_base += D.n_columns;
        uni_base += D.n_columns * D.n_uni_z;
        lj_base += d.n_lj_types * d.n_lj_types;
        sd[k] = D;
    }
    sys_col_base[S] = col_base;
    // the j-queue and j-list kernels read the LJ table pre-scaled for forces, (6 C6, 12 C12),
    // from a copy after the plain one
    for (int k = 0; k < S; k++) sd[k].ljf_off = lj_base;
    for (int i = 0; i < lj_base; i++) lj.push_back(make_float2(6.0f * lj[i].x, 12.0f * lj[i].y));
    e->n_atoms = atom_base;
    e->n_cols = col_base;
    e->n_uni = uni_base;
    e->cells_cap = cells_cap;
    e->slots_cap = cells_cap * OG_CELL;
    e->nnc = nnc;
    e->n_excess = (int)excess.size();
    e->n_bonds = (int)bondv.size();
    e->n_angles = (int)anglev.size();
    e->n_spair = (int)spair.size();
    e->n_strio = (int)strio.size();
    e->n_tors = (int)torsv.size();
    e->n_impro = (int)improv.size();
    e->n_nb14 = (int)nb14v.size();
    e->n_squad = (int)squadv.size();
    e->n_groups = (int)grp_mass_inv.size();
    e->any_groups = e->n_groups > 0;
    // ---- allocation + upload
    std::vector<SysDev> sdv(sd);
    if ((s = upload(e, &e->d_sys, sdv)) || (s = dalloc(e, &e->d_counters, OG_CNT_SIZE)) ||
        (s = dalloc(e, &e->d_step, 1)) || (s = dalloc(e, &e->d_trace_count, 1)) || (s = upload(e, &e->d_crd, crd)) ||
        (s = dalloc(e, &e->d_crd_prev, crd.size())) || (s = dalloc(e, &e->d_vel, crd.size())) ||
        (s = upload(e, &e->d_vel_next, vel)) || (s = dalloc(e, &e->d_work, crd.size())) ||
        (s = dalloc(e, &e->d_buf_crd, crd.size())) || (s = upload(e, &e->d_charge, charge)) ||
        (s = dalloc(e, &e->d_ke, e->n_atoms)) || (s = upload(e, &e->d_charge_f, charge_f)) ||
        (s = upload(e, &e->d_mass, mass)) || (s = upload(e, &e->d_mass_inv, mass_inv)) ||
        (s = upload(e, &e->d_atom_type, atom_type)) || (s = upload(e, &e->d_atom_sys, atom_sys)) ||
        (s = dalloc(e, &e->d_atom_col, e->n_atoms)) || (s = dalloc(e, &e->d_atom_slot, e->n_atoms)) ||
        (s = upload(e, &e->d_atom_group, atom_group)) || (s = dalloc(e, &e->d_atom_key, e->n_atoms)) ||
        (s = dalloc(e, &e->d_col_keys, e->n_atoms)) || (s = dalloc(e, &e->d_col_count, e->n_cols)) ||
        (s = dalloc(e, &e->d_col_fill, e->n_cols)) || (s = dalloc(e, &e->d_col_atom_start, e->n_cols + 1)) ||
        (s = dalloc(e, &e->d_col_cell_start, e->n_cols + 1)) || (s = dalloc(e, &e->d_col_head_cell, e->n_cols + 1)) ||
        (s = upload(e, &e->d_col_sys, col_sys)) || (s = upload(e, &e->d_sys_col_base, sys_col_base)) ||
        (s = dalloc(e, &e->d_sys_cell_base, S + 1)) || (s = dalloc(e, &e->d_cell_col, cells_cap)) ||
        (s = dalloc(e, &e->d_cell_sys, cells_cap)) || (s = dalloc(e, &e->d_cp_head, cells_cap + 1)) ||
        (s = dalloc(e, &e->d_cell_origin, 3 * (size_t)cells_cap)) ||
        (s = dalloc(e, &e->d_cell_acc, OG_CELL_ACC * (size_t)cells_cap)) || (s = dalloc(e, &e->d_cell_zr, cells_cap)) ||
        (s = dalloc(e, &e->d_cell_uni, cells_cap)) || (s = dalloc(e, &e->d_cell_valid, cells_cap)) ||
        (s = dalloc(e, &e->d_bbox, 2 * (size_t)cells_cap)) ||
        (s = dalloc(e, &e->d_slot_atom, e->slots_cap)) || (s = dalloc(e, &e->d_slot_type, e->slots_cap)) ||
        (s = dalloc(e, &e->d_slot_crd, 3 * (size_t)e->slots_cap)) || (s = dalloc(e, &e->d_xq, e->slots_cap)) ||
        (e->list_policy == OG_LIST_DISPLACEMENT && (s = dalloc(e, &e->d_xq_build, e->slots_cap))) ||
        (s = dalloc(e, &e->d_frc, 3 * (size_t)e->slots_cap)) || (s = dalloc(e, &e->d_uni_lo, e->n_uni)) ||
        (s = dalloc(e, &e->d_uni_hi, e->n_uni)) || (s = upload(e, &e->d_excl_start, excl_start)) ||
        (s = upload(e, &e->d_excl_list, excl_list)) || (s = upload(e, &e->d_excess, excess)) ||
        (s = upload(e, &e->d_excess_sys, excess_sys)) || (s = dalloc(e, &e->d_e_exc, excess.size())) ||
        (s = upload(e, &e->d_bond, bondv)) || (s = upload(e, &e->d_bond_sys, bond_sys)) ||
        (s = upload(e, &e->d_bond_kr, bond_kr)) || (s = dalloc(e, &e->d_e_bond, bondv.size())) ||
        (s = upload(e, &e->d_angle, anglev)) || (s = upload(e, &e->d_angle_kt, angle_kt)) ||
        (s = dalloc(e, &e->d_e_angle, anglev.size())) || (s = upload(e, &e->d_spair, spair)) ||
        (s = upload(e, &e->d_spair_sys, spair_sys)) || (s = upload(e, &e->d_spair_d2, spair_d2)) ||
        (s = upload(e, &e->d_strio, strio)) || (s = upload(e, &e->d_strio_d2, strio_d2)) ||
        (s = upload(e, &e->d_tors, torsv)) || (s = upload(e, &e->d_tors_p, tors_p)) ||
        (s = upload(e, &e->d_tors_sys, tors_sys)) || (s = dalloc(e, &e->d_e_tors, torsv.size())) ||
        (s = upload(e, &e->d_impro, improv)) || (s = upload(e, &e->d_impro_p, impro_p)) ||
        (s = upload(e, &e->d_impro_sys, impro_sys)) || (s = dalloc(e, &e->d_e_impro, improv.size())) ||
        (s = upload(e, &e->d_nb14, nb14v)) || (s = upload(e, &e->d_nb14_t, nb14t)) ||
        (s = upload(e, &e->d_nb14_c, nb14c)) || (s = upload(e, &e->d_nb14_sys, nb14_sys)) ||
        (s = dalloc(e, &e->d_e_nb14, 2 * nb14v.size())) || (s = upload(e, &e->d_squad, squadv)) ||
        (s = upload(e, &e->d_squad_d2, squad_d2)) || (s = upload(e, &e->d_squad_sys, squad_sys)) ||
        (s = upload(e, &e->d_grp_start, grp_start)) || (s = upload(e, &e->d_grp_atoms, grp_atoms)) ||
        (s = upload(e, &e->d_grp_sys, grp_sys)) || (s = upload(e, &e->d_grp_mass_inv, grp_mass_inv)) ||
        (s = dalloc(e, &e->d_moment, 3 * (size_t)(e->n_groups + 1))) || (s = upload(e, &e->d_lj, lj)) ||
        (s = upload(e, &e->d_hps, hps_tab)) || (s = upload(e, &e->d_ele, ele_tab)) ||
        (!lj64.empty() && (s = upload(e, &e->d_lj64, lj64))) ||
        (s = dalloc(e, &e->d_sys_acc, OG_ACC_SIZE * (size_t)S)) || (s = dalloc(e, &e->d_mcmd, S)) ||
        (s = dalloc(e, &e->d_energies, OG_N_ENERGY * (size_t)S)) || (s = upload(e, &e->d_thermo, thermo)) ||
        (s = dalloc(e, &e->d_sum_tmp, S)) || (s = upload(e, &e->d_mask_plain, mask_plain)) ||
        (s = upload(e, &e->d_mask_thermo, mask_thermo)) || (s = dalloc(e, &e->d_active, S)) ||
        (s = dalloc(e, &e->d_any, 1)) || (s = dalloc(e, &e->d_thermo_it, 1)) ||
        (s = dalloc(e, &e->d_sys_fault, S)) || (s = dalloc(e, &e->d_snap_ctr, 2)) ||
        (s = dalloc(e, &e->d_cell_excl, (size_t)OG_CELL_EXCL * cells_cap)))
        return s;
    // V-McMD: a ring of log entries per slot, long enough for one list interval of entries, so
    // that og_step can drain it between graph replays
    e->n_vm = (int)e->vm_sys.size();
    e->vm_log_cap = std::max(4096, e->intvl + 2);
    e->vm.assign(e->n_vm, VmLog{});
    for (int m = 0; m < e->n_vm; m++) {
        const SysDev &D = sd[e->vm_sys[m]];
        // the first entries this engine writes: steps k * interval >= first_step, k >= 1
        e->vm[m].vs_next_k = std::max(1LL, (D.first_step + D.vs_trans_intvl - 1) / D.vs_trans_intvl);
        if (D.vs_lambda_intvl > 0)
            e->vm[m].lam_next_k = std::max(1LL, (D.first_step + D.vs_lambda_intvl - 1) / D.vs_lambda_intvl);
    }
    // trajectory frames: the first frame this engine writes is labelled k * interval with
    // k * interval - 1 >= first_step
    e->n_tr = (int)e->tr_sys.size();
    e->n_tr_entries = (int)tr_atom.size();
    e->tr.assign(e->n_tr, TrLog{});
    for (int m = 0; m < e->n_tr; m++) {
        const SysDev &D = sd[e->tr_sys[m]];
        e->tr[m].next_k = (D.first_step + D.tr_interval) / D.tr_interval;
    }
    logs_update_limit(e);
    if ((s = upload(e, &e->d_vstates, vstates)) || (s = upload(e, &e->d_vs_cur, vs_cur)) ||
        (s = dalloc(e, &e->d_vm_snap_cur, S)) || (s = upload(e, &e->d_mt, mt_all)) ||
        (s = dalloc(e, &e->d_vm_snap_mt, mt_all.size())) ||
        (s = dalloc(e, &e->d_vs_log, (size_t)e->n_vm * e->vm_log_cap)) ||
        (s = dalloc(e, &e->d_lambda_log, (size_t)e->n_vm * e->vm_log_cap)) ||
        (s = upload(e, &e->d_tr_atom, tr_atom)) || (s = upload(e, &e->d_tr_sys, tr_sysv)) ||
        (s = upload(e, &e->d_tr_idx, tr_idx)) || (s = dalloc(e, &e->d_frames, (size_t)tr_crd_total)) ||
        (s = dalloc(e, &e->d_frame_ene, (size_t)tr_ene_total)))
        return s;
    {
        std::vector<int> sa(S + 1), se(S + 1), sb(S + 1), sg(S + 1), st(S + 1), si(S + 1), s14(S + 1);
        int ma = 1, mcl = 1, me = 1, mb = 1, mg = 1, mt = 1, mi = 1, m14 = 1;
        for (int k = 0; k < S; k++) {
            const SysDev &D = sd[k];
            sa[k] = D.atom_base;
            se[k] = D.excess_base;
            sb[k] = D.bond_base;
            sg[k] = D.angle_base;
            st[k] = D.tors_base;
            si[k] = D.impro_base;
            s14[k] = D.nb14_base;
            auto ch = [](long long n) { return (int)((n + 4095) / 4096); };
            mt = std::max(mt, ch(D.n_tors));
            mi = std::max(mi, ch(D.n_impro));
            m14 = std::max(m14, ch(D.n_nb14));
            ma = std::max(ma, ch(D.n_atoms));
            mcl = std::max(mcl, ch(D.n_atoms / OG_CELL + D.n_columns + 1));
            me = std::max(me, ch(D.n_excess));
            mb = std::max(mb, ch(D.n_bonds));
            mg = std::max(mg, ch(D.n_angles));
        }
        sa[S] = e->n_atoms;
        se[S] = (int)excess.size();
        sb[S] = (int)bondv.size();
        sg[S] = (int)anglev.size();
        st[S] = (int)torsv.size();
        si[S] = (int)improv.size();
        s14[S] = (int)nb14v.size();
        e->mc_tors = mt;
        e->mc_impro = mi;
        e->mc_nb14 = m14;
        int mgr = 1;
        for (int g = 0; g < e->n_groups; g++) mgr = std::max(mgr, (grp_start[g + 1] - grp_start[g] + 4095) / 4096);
        e->mc_atoms = ma;
        e->mc_cells = mcl;
        e->mc_exc = me;
        e->mc_bond = mb;
        e->mc_angle = mg;
        e->mc_grp = mgr;
        size_t part = (size_t)S *
                      std::max(std::max(std::max(ma, mcl), std::max(me, std::max(mb, mg))),
                               std::max(mt, std::max(mi, m14))) * 10;
        part = std::max(part, (size_t)(e->n_groups + 1) * mgr * 3);
        if ((s = upload(e, &e->d_seg_atoms, sa)) || (s = upload(e, &e->d_seg_exc, se)) ||
            (s = upload(e, &e->d_seg_bond, sb)) || (s = upload(e, &e->d_seg_angle, sg)) ||
            (s = upload(e, &e->d_seg_tors, st)) || (s = upload(e, &e->d_seg_impro, si)) ||
            (s = upload(e, &e->d_seg_nb14, s14)) ||
            (s = dalloc(e, &e->d_part, part)))
            return s;
    }
    const long long n_items = (long long)cells_cap * nnc + 1;
    if ((s = dalloc(e, &e->d_count, n_items)) || (s = dalloc(e, &e->d_offset, n_items))) return s;
    for (long long len = n_items; len > 1;) {
        long long nb = (len + 2047) / 2048;
        long long *a, *b;
        if ((s = dalloc(e, &a, nb)) || (s = dalloc(e, &b, nb))) return s;
        e->d_scan_tmp.push_back(a);
        e->d_scan_tmp.push_back(b);
        len = nb;
    }
    CK(cudaMemsetAsync(e->d_counters, 0, sizeof(int) * OG_CNT_SIZE, e->stream));
    CK(cudaMemsetAsync(e->d_step, 0, sizeof(long long), e->stream));
    CK(cudaMemsetAsync(e->d_trace_count, 0, sizeof(long long), e->stream));
    CK(cudaMemsetAsync(e->d_count + (n_items - 1), 0, sizeof(int), e->stream));
    CK(cudaMemsetAsync(e->d_frc, 0, sizeof(unsigned long long) * 3 * (size_t)e->slots_cap, e->stream));
    CK(cudaMemsetAsync(e->d_cell_acc, 0, sizeof(double) * OG_CELL_ACC * (size_t)cells_cap, e->stream));
    CK(cudaMemsetAsync(e->d_sys_acc, 0, sizeof(double) * OG_ACC_SIZE * S, e->stream));
    CK(cudaMemsetAsync(e->d_slot_crd, 0, sizeof(double) * 3 * (size_t)e->slots_cap, e->stream));
    if ((s = grow_pairs(e, (long long)cells_cap * 180))) return s;
    e->finalized = true;
    e->host_step = 0;
    // initial list + forces (DynamicsMode::initial_preprocess -> calc_energy_force)
    if ((s = build_list_checked(e))) return s;
    if ((s = autotune_pair(e))) return s;
    if ((s = compute_forces(e, false))) return s;
    CK(cudaStreamSynchronize(e->stream));
    return check_flags(e);
}

og_status og_step(og_engine *e, int32_t n_steps) {
    if (!e) return OG_ERR_INVALID;
    if (!e->finalized) return fail(e, OG_ERR_STATE, "og_step before og_finalize");
    if (n_steps < 0) return fail(e, OG_ERR_INVALID, "negative step count");
    CK(cudaSetDevice(e->device));
    og_status s;
    e->launches = 0;
    e->faults.clear();
    const long long builds0 = e->builds_seen;
    if (e->timing) {
        e->pair_ms = 0.0;
    }
    // snapshot for a capacity retry: crd, vel_next and the step counters
    if (!e->d_snap && (s = dalloc(e, &e->d_snap, 6 * (size_t)e->n_atoms))) return s;
    const long long step0 = e->host_step;
    // V-McMD log positions at the call's start, for an undo
    struct VmMark {
        long long vs_k, lam_k;
        size_t vs_n, lam_n;
    };
    std::vector<VmMark> vm0(e->n_vm);
    for (int m = 0; m < e->n_vm; m++)
        vm0[m] = {e->vm[m].vs_next_k, e->vm[m].lam_next_k, e->vm[m].vs.size(), e->vm[m].lam.size()};
    std::vector<VmMark> tr0(e->n_tr);  // trajectory: next frame and frames held
    for (int m = 0; m < e->n_tr; m++) tr0[m] = {e->tr[m].next_k, 0, e->tr[m].step.size(), 0};
    for (int attempt = 0; attempt < 3; attempt++) {
        if (e->n_vm) {
            CK(cudaMemcpyAsync(e->d_vm_snap_cur, e->d_vs_cur, sizeof(int) * e->n_sys, cudaMemcpyDeviceToDevice,
                               e->stream));
            CK(cudaMemcpyAsync(e->d_vm_snap_mt, e->d_mt, sizeof(unsigned) * OG_MT_WORDS * e->n_vm,
                               cudaMemcpyDeviceToDevice, e->stream));
        }
        CK(cudaMemcpyAsync(e->d_snap, e->d_crd, sizeof(double) * 3 * e->n_atoms, cudaMemcpyDeviceToDevice, e->stream));
        CK(cudaMemcpyAsync(e->d_snap + 3 * (size_t)e->n_atoms, e->d_vel_next, sizeof(double) * 3 * e->n_atoms,
                           cudaMemcpyDeviceToDevice, e->stream));
        CK(cudaMemcpyAsync(e->d_snap_ctr, e->d_step, sizeof(long long), cudaMemcpyDeviceToDevice, e->stream));
        CK(cudaMemcpyAsync(e->d_snap_ctr + 1, e->d_trace_count, sizeof(long long), cudaMemcpyDeviceToDevice,
                           e->stream));
        if ((s = clear_flags(e))) return s;
        e->pev_used = 0;
        e->host_cond_builds = 0;
        if (e->timing) CK(cudaEventRecord(e->ev_step0, e->stream));
        for (int i = 0; i < n_steps;) {
            // whole list intervals replay the captured graph (not while per-kernel timing is on)
            if (e->use_graphs && e->timing != 1 && e->host_step % e->intvl == 0 && n_steps - i >= e->intvl) {
                if ((s = logs_reserve(e, e->intvl))) return s;
                if (!e->graph_exec && (s = capture_interval(e))) return s;
                if (e->graph_exec) {
                    CK(cudaGraphLaunch(e->graph_exec, e->stream));
                    e->launches += e->graph_kernels;
                    e->graph_replays++;
                    e->host_step += e->intvl;
                    i += e->intvl;
                    continue;
                }
            }
            if ((s = logs_reserve(e, 1))) return s;
            if ((s = run_step(e, i == n_steps - 1))) return s;
            i++;
        }
        if (e->timing) {
            CK(cudaEventRecord(e->ev_step1, e->stream));
            CK(cudaEventSynchronize(e->ev_step1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, e->ev_step0, e->ev_step1));
            e->step_ms = ms;
            e->pair_ms = 0.0;
            for (int i = 0; i < e->pev_used; i++) {
                CK(cudaEventElapsedTime(&ms, e->pev0[i], e->pev1[i]));
                e->pair_ms += ms;
            }
        }
        int c[OG_CNT_SIZE];
        if ((s = read_counters(e, c))) return s;
        // list builds that ran as conditional nodes of graph replays (the displacement policy)
        if (e->list_policy == OG_LIST_DISPLACEMENT)
            e->launches += std::max(0LL, c[OG_CNT_LIST_BUILDS] - builds0 - e->host_cond_builds) * e->cond_build_kernels;
        const int f = c[OG_CNT_FLAGS];
        const bool fault = (f & (OG_FLAG_BAD_COORD | OG_FLAG_COLUMN_CAPACITY | OG_FLAG_DISPLACEMENT)) != 0;
        if (!fault && !(f & OG_FLAG_PAIR_CAPACITY)) return check_flags(e);
        if (fault) {
            // A system left its box or packed a column beyond capacity.  Systems are
            // independent, so the others are sound; the call is undone for all of them and the
            // faulted systems are named, for the caller to drop them and step the rest again.
            e->faults.assign(e->n_sys, 0);
            CK(cudaMemcpy(e->faults.data(), e->d_sys_fault, sizeof(int) * e->n_sys, cudaMemcpyDeviceToHost));
        } else if ((s = grow_pairs(e, (long long)c[OG_CNT_N_PAIRS] * 5 / 4))) {
            return s;
        }
        // restore the state of the call's start (and redo it after a capacity miss)
        CK(cudaMemcpyAsync(e->d_crd, e->d_snap, sizeof(double) * 3 * e->n_atoms, cudaMemcpyDeviceToDevice, e->stream));
        CK(cudaMemcpyAsync(e->d_vel_next, e->d_snap + 3 * (size_t)e->n_atoms, sizeof(double) * 3 * e->n_atoms,
                           cudaMemcpyDeviceToDevice, e->stream));
        CK(cudaMemcpyAsync(e->d_step, e->d_snap_ctr, sizeof(long long), cudaMemcpyDeviceToDevice, e->stream));
        CK(cudaMemcpyAsync(e->d_trace_count, e->d_snap_ctr + 1, sizeof(long long), cudaMemcpyDeviceToDevice,
                           e->stream));
        if (e->n_vm) {
            CK(cudaMemcpyAsync(e->d_vs_cur, e->d_vm_snap_cur, sizeof(int) * e->n_sys, cudaMemcpyDeviceToDevice,
                               e->stream));
            CK(cudaMemcpyAsync(e->d_mt, e->d_vm_snap_mt, sizeof(unsigned) * OG_MT_WORDS * e->n_vm,
                               cudaMemcpyDeviceToDevice, e->stream));
            for (int m = 0; m < e->n_vm; m++) {
                VmLog &L = e->vm[m];
                L.vs_next_k = vm0[m].vs_k;
                L.lam_next_k = vm0[m].lam_k;
                L.vs.resize(vm0[m].vs_n);
                L.vs_step.resize(vm0[m].vs_n);
                L.lam.resize(vm0[m].lam_n);
                L.lam_step.resize(vm0[m].lam_n);
            }
        }
        for (int m = 0; m < e->n_tr; m++) {
            TrLog &T = e->tr[m];
            const size_t fc = 3 * (size_t)e->sys[e->tr_sys[m]].dev.tr_n;
            T.next_k = tr0[m].vs_k;
            T.step.resize(tr0[m].vs_n);
            T.crd.resize(tr0[m].vs_n * fc);
            T.ene.resize(tr0[m].vs_n * OG_N_ENERGY);
        }
        CK(cudaStreamSynchronize(e->stream));
        e->host_step = step0;
        logs_update_limit(e);
        // the list must be rebuilt from the restored coordinates before the first step: under
        // the displacement policy it is marked stale (the next step builds it); under the fixed
        // schedule it is built now unless the step is a rebuild step anyway.  A faulted system's
        // restored coordinates may not bin (the caller placed them, or they are those the fault
        // ran from): a failed build then leaves valid indices, and the call reports the fault.
        if (e->list_policy == OG_LIST_DISPLACEMENT) {
            CK(cudaMemsetAsync(e->d_counters + OG_CNT_LIST_STALE, 1, sizeof(int), e->stream));
        } else if (step0 % e->intvl != 0) {
            s = build_list_checked(e);
            if (s && !fault) return s;
        }
        if (fault) {
            std::string who;
            for (int k = 0; k < e->n_sys; k++)
                if (e->faults[k]) who += (who.empty() ? "" : ", ") + std::to_string(k);
            return fail(e, OG_ERR_SYSTEM_FAULT, "system(s) %s faulted (non-finite or far out-of-box coordinate, a "
                        "one-step displacement beyond the list margin, or a column beyond %d atoms); all systems "
                        "are back at the call's start", who.c_str(), OG_MAX_COLUMN_ATOMS);
        }
    }
    return fail(e, OG_ERR_CAPACITY, "cell-pair list kept overflowing");
}

og_status og_compute_forces(og_engine *e) {
    if (!e) return OG_ERR_INVALID;
    if (!e->finalized) return fail(e, OG_ERR_STATE, "og_compute_forces before og_finalize");
    CK(cudaSetDevice(e->device));
    og_status s = build_list_checked(e);
    if (s) return s;
    // forces of the current list: the accumulators are clear after every collect
    if ((s = compute_forces(e, true))) return s;
    CK(cudaStreamSynchronize(e->stream));
    return check_flags(e);
}

og_status og_compute_forces_current(og_engine *e) {
    if (!e) return OG_ERR_INVALID;
    if (!e->finalized) return fail(e, OG_ERR_STATE, "og_compute_forces_current before og_finalize");
    CK(cudaSetDevice(e->device));
    og_status s = clear_flags(e);
    if (s) return s;
    if ((s = compute_forces(e, true))) return s;
    CK(cudaStreamSynchronize(e->stream));
    return check_flags(e);
}

og_status og_set_pair_only(og_engine *e, int32_t on) {
    if (!e) return OG_ERR_INVALID;
    if (e->finalized) return fail(e, OG_ERR_STATE, "og_set_pair_only after og_finalize");
    e->pair_only = on != 0;
    return OG_OK;
}

og_status og_set_state(og_engine *e, int32_t sys, const double *crd, const double *vel_next) {
    if (!e || !e->finalized) return fail(e, OG_ERR_STATE, "og_set_state before og_finalize");
    if (sys < 0 || sys >= e->n_sys) return fail(e, OG_ERR_INVALID, "bad system id");
    const SysDev &D = e->sys[sys].dev;
    if (crd)
        CK(cudaMemcpyAsync(e->d_crd + 3 * (size_t)D.atom_base, crd, sizeof(double) * 3 * D.n_atoms,
                           cudaMemcpyHostToDevice, e->stream));
    if (vel_next)
        CK(cudaMemcpyAsync(e->d_vel_next + 3 * (size_t)D.atom_base, vel_next, sizeof(double) * 3 * D.n_atoms,
                           cudaMemcpyHostToDevice, e->stream));
    if (crd && e->list_policy == OG_LIST_DISPLACEMENT)
        CK(cudaMemsetAsync(e->d_counters + OG_CNT_LIST_STALE, 1, sizeof(int), e->stream));
    CK(cudaStreamSynchronize(e->stream));
    // new coordinates invalidate the grid: rebuild at the next step
    if (crd) e->host_step = ((e->host_step + e->intvl - 1) / e->intvl) * e->intvl;
    if (crd && e->host_step % e->intvl != 0) return build_list_checked(e);
    if (crd) {
        long long st = e->host_step;
        CK(cudaMemcpyAsync(e->d_step, &st, sizeof(long long), cudaMemcpyHostToDevice, e->stream));
        CK(cudaStreamSynchronize(e->stream));
    }
    return OG_OK;
}

og_status og_get_state(og_engine *e, int32_t sys, double *crd, double *vel_next) {
    if (!e || !e->finalized) return fail(e, OG_ERR_STATE, "og_get_state before og_finalize");
    if (sys < 0 || sys >= e->n_sys) return fail(e, OG_ERR_INVALID, "bad system id");
    const SysDev &D = e->sys[sys].dev;
    if (crd)
        CK(cudaMemcpyAsync(crd, e->d_crd + 3 * (size_t)D.atom_base, sizeof(double) * 3 * D.n_atoms,
                           cudaMemcpyDeviceToHost, e->stream));
    if (vel_next)
        CK(cudaMemcpyAsync(vel_next, e->d_vel_next + 3 * (size_t)D.atom_base, sizeof(double) * 3 * D.n_atoms,
                           cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    return OG_OK;
}

og_status og_get_forces(og_engine *e, int32_t sys, double *work, double *energies, double *virial) {
    if (!e || !e->finalized) return fail(e, OG_ERR_STATE, "og_get_forces before og_finalize");
    if (sys < 0 || sys >= e->n_sys) return fail(e, OG_ERR_INVALID, "bad system id");
    const SysDev &D = e->sys[sys].dev;
    if (work)
        CK(cudaMemcpyAsync(work, e->d_work + 3 * (size_t)D.atom_base, sizeof(double) * 3 * D.n_atoms,
                           cudaMemcpyDeviceToHost, e->stream));
    double acc[OG_ACC_SIZE];
    CK(cudaMemcpyAsync(acc, e->d_sys_acc + OG_ACC_SIZE * sys, sizeof(acc), cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    if (energies) {
        for (int q = 0; q < OG_N_ENERGY; q++) energies[q] = 0.0;
        energies[OG_E_VDW] = acc[OG_ACC_VDW];
        energies[OG_E_ELE] = acc[OG_ACC_ELE] + acc[OG_ACC_EXCESS] + D.self_energy;
        energies[OG_E_BOND] = acc[OG_ACC_BOND];
        energies[OG_E_ANGLE] = acc[OG_ACC_ANGLE];
        energies[OG_E_TORSION] = acc[OG_ACC_TORSION];
        energies[OG_E_IMPROPER] = acc[OG_ACC_IMPRO];
        energies[OG_E_VDW14] = acc[OG_ACC_VDW14];
        energies[OG_E_ELE14] = acc[OG_ACC_ELE14];
        energies[OG_E_POTENTIAL] = energies[OG_E_VDW] + energies[OG_E_ELE] + energies[OG_E_BOND] + energies[OG_E_ANGLE] +
                                   energies[OG_E_TORSION] + energies[OG_E_IMPROPER] + energies[OG_E_VDW14] +
                                   energies[OG_E_ELE14];
        energies[OG_E_ELE_EXCESS] = acc[OG_ACC_EXCESS];
        energies[OG_E_ELE_SELF] = D.self_energy;
    }
    if (virial)
        for (int q = 0; q < 9; q++) virial[q] = acc[OG_ACC_VIR + q];
    return OG_OK;
}

og_status og_get_energies(og_engine *e, int32_t sys, double *energies) {
    if (!e || !e->finalized) return fail(e, OG_ERR_STATE, "og_get_energies before og_finalize");
    if (sys < 0 || sys >= e->n_sys || !energies) return fail(e, OG_ERR_INVALID, "bad arguments");
    CK(cudaMemcpyAsync(energies, e->d_energies + OG_N_ENERGY * (size_t)sys, sizeof(double) * OG_N_ENERGY,
                       cudaMemcpyDeviceToHost, e->stream));
    CK(cudaStreamSynchronize(e->stream));
    return OG_OK;
}

og_status og_get_grid_info(og_engine *e, int32_t sys, int32_t *n_cells, int32_t *n_columns, int32_t *n_pairs) {
    if (!e || !e->finalized) return fail(e, OG_ERR_STATE, "og_get_grid_info before og_finalize");
    if (sys < 0 || sys >= e->n_sys) return fail(e, OG_ERR_INVALID, "bad system id");
    std::vector<int> base(e->n_sys + 1);
    CK(cudaMemcpyAsync(base.data(), e->d_sys_cell_base, sizeof(int) * (e->n_sys + 1), cudaMemcpyDeviceToHost,
                       e->stream));
    CK(cudaStreamSynchronize(e->stream));
    int h0 = 0, h1 = 0;
    CK(cudaMemcpy(&h0, e->d_cp_head + base[sys], sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&h1, e->d_cp_head + base[sys + 1], sizeof(int), cudaMemcpyDeviceToHost));
    if (n_cells) *n_cells = base[sys + 1] - base[sys];
    if (n_columns) *n_columns = e->sys[sys].dev.n_columns;
    if (n_pairs) *n_pairs = h1 - h0;
    return OG_OK;
}

og_status og_get_grid(og_engine *e, int32_t sys, int32_t *slot_atomid, double *slot_crd, int32_t *col_head_cell) {
    int32_t nc = 0, ncol = 0, np = 0;
    og_status s = og_get_grid_info(e, sys, &nc, &ncol, &np);
    if (s) return s;
    std::vector<int> base(e->n_sys + 1);
    CK(cudaMemcpy(base.data(), e->d_sys_cell_base, sizeof(int) * (e->n_sys + 1), cudaMemcpyDeviceToHost));
    const SysDev &D = e->sys[sys].dev;
    const size_t s0 = (size_t)base[sys] * OG_CELL, ns = (size_t)nc * OG_CELL;
    if (slot_atomid) {
        CK(cudaMemcpy(slot_atomid, e->d_slot_atom + s0, sizeof(int) * ns, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < ns; i++)
            if (slot_atomid[i] >= 0) slot_atomid[i] -= D.atom_base;
    }
    if (slot_crd) CK(cudaMemcpy(slot_crd, e->d_slot_crd + 3 * s0, sizeof(double) * 3 * ns, cudaMemcpyDeviceToHost));
    if (col_head_cell) {
        CK(cudaMemcpy(col_head_cell, e->d_col_head_cell + D.col_base, sizeof(int) * D.n_columns,
                      cudaMemcpyDeviceToHost));
        for (int c = 0; c < D.n_columns; c++)
            if (col_head_cell[c] >= 0) col_head_cell[c] -= base[sys];
        col_head_cell[D.n_columns] = nc;
    }
    return OG_OK;
}

og_status og_get_cell_pairs(og_engine *e, int32_t sys, int32_t *idx_head, int32_t *cell1, int32_t *cell2,
                            int32_t *image, uint64_t *mask) {
    int32_t nc = 0, ncol = 0, np = 0;
    og_status s = og_get_grid_info(e, sys, &nc, &ncol, &np);
    if (s) return s;
    std::vector<int> base(e->n_sys + 1);
    CK(cudaMemcpy(base.data(), e->d_sys_cell_base, sizeof(int) * (e->n_sys + 1), cudaMemcpyDeviceToHost));
    std::vector<int> head(nc + 1);
    CK(cudaMemcpy(head.data(), e->d_cp_head + base[sys], sizeof(int) * (nc + 1), cudaMemcpyDeviceToHost));
    const int p0 = head[0];
    std::vector<int2> ci(np);
    if (np) CK(cudaMemcpy(ci.data(), e->d_cp_c2img + p0, sizeof(int2) * np, cudaMemcpyDeviceToHost));
    if (mask && np) CK(cudaMemcpy(mask, e->d_cp_mask + p0, sizeof(uint64_t) * np, cudaMemcpyDeviceToHost));
    for (int c = 0; c <= nc; c++)
        if (idx_head) idx_head[c] = head[c] - p0;
    for (int c = 0; c < nc; c++)
        for (int k = head[c]; k < head[c + 1]; k++) {
            if (cell1) cell1[k - p0] = c;
            if (cell2) cell2[k - p0] = ci[k - p0].x - base[sys];
            if (image) image[k - p0] = ci[k - p0].y;
        }
    return OG_OK;
}

og_status og_set_trace(og_engine *e, int32_t capacity) {
    if (!e || !e->finalized) return fail(e, OG_ERR_STATE, "og_set_trace before og_finalize");
    if (capacity < 0) return fail(e, OG_ERR_INVALID, "negative capacity");
    drop_graph(e);  // the graph holds the trace buffer and its capacity
    if (e->d_trace) {
        dfree(e, e->d_trace);
        e->d_trace = nullptr;
    }
    e->trace_cap = capacity;
    if (capacity > 0) {
        og_status s = dalloc(e, &e->d_trace, (size_t)capacity * e->n_sys * OG_N_ENERGY);
        if (s) return s;
    }
    CK(cudaMemsetAsync(e->d_trace_count, 0, sizeof(long long), e->stream));
    CK(cudaStreamSynchronize(e->stream));
    return OG_OK;
}

og_status og_get_trace(og_engine *e, double *out, int32_t max_steps, int32_t *n_out) {
    if (!e || !e->finalized) return fail(e, OG_ERR_STATE, "og_get_trace before og_finalize");
    long long cnt = 0;
    CK(cudaMemcpy(&cnt, e->d_trace_count, sizeof(long long), cudaMemcpyDeviceToHost));
    if (e->trace_cap <= 0) {
        if (n_out) *n_out = 0;
        return OG_OK;
    }
    long long avail = cnt < e->trace_cap ? cnt : e->trace_cap;
    long long first = cnt - avail;
    int n = (int)(avail < max_steps ? avail : max_steps);
    const size_t row = (size_t)e->n_sys * OG_N_ENERGY;
    std::vector<double> all((size_t)e->trace_cap * row);
    CK(cudaMemcpy(all.data(), e->d_trace, sizeof(double) * all.size(), cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; i++) {
        long long r = (first + i) % e->trace_cap;
        memcpy(out + i * row, all.data() + r * row, sizeof(double) * row);
    }
    if (n_out) *n_out = n;
    return OG_OK;
}

og_status og_get_stats(og_engine *e, int64_t *kernel_launches, double *pair_kernel_ms, double *step_ms) {
    if (!e) return OG_ERR_INVALID;
    if (kernel_launches) *kernel_launches = e->launches;
    if (pair_kernel_ms) *pair_kernel_ms = e->pair_ms;
    if (step_ms) *step_ms = e->step_ms;
    return OG_OK;
}

og_status og_get_sizes(og_engine *e, int32_t *n_systems, int64_t *n_atoms_total) {
    if (!e) return OG_ERR_INVALID;
    if (n_systems) *n_systems = (int32_t)e->sys.size();
    if (n_atoms_total) {
        int64_t t = 0;
        for (auto &h : e->sys) t += h.d.n_atoms;
        *n_atoms_total = t;
    }
    return OG_OK;
}

og_status og_get_vmcmd_state(og_engine *e, int32_t sys, int32_t *cur_vs, uint32_t *mt_state) {
    if (!e || !e->finalized) return fail(e, OG_ERR_STATE, "og_get_vmcmd_state before og_finalize");
    if (sys < 0 || sys >= e->n_sys) return fail(e, OG_ERR_INVALID, "bad system id");
    const SysDev &D = e->sys[sys].dev;
    if (D.n_vs == 0) return fail(e, OG_ERR_INVALID, "system %d has no V-McMD", sys);
    if (cur_vs) CK(cudaMemcpyAsync(cur_vs, e->d_vs_cur + sys, sizeof(int32_t), cudaMemcpyDeviceToHost, e->stream));
    if (mt_state) {
        if (D.vm_slot < 0) return fail(e, OG_ERR_INVALID, "system %d has one virtual state and no generator", sys);
        CK(cudaMemcpyAsync(mt_state, e->d_mt + (size_t)OG_MT_WORDS * D.vm_slot, sizeof(uint32_t) * OG_MT_WORDS,
                           cudaMemcpyDeviceToHost, e->stream));
    }
    CK(cudaStreamSynchronize(e->stream));
    return OG_OK;
}


og_status og_take_vs_log(og_engine *e, int32_t sys, int64_t max, int64_t *step, int32_t *vs, int64_t *n) {
    return vm_take<int32_t>(e, sys, max, step, vs, n, true);
}

og_status og_take_lambda_log(og_engine *e, int32_t sys, int64_t max, int64_t *step, double *lambda, int64_t *n) {
    return vm_take<double>(e, sys, max, step, lambda, n, false);
}

og_status og_set_trajectory(og_engine *e, int32_t sys, int32_t interval, const int32_t *group_atoms,
                            int32_t n_group) {
    if (!e) return OG_ERR_INVALID;
    if (e->finalized) return fail(e, OG_ERR_STATE, "og_set_trajectory after og_finalize");
    if (sys < 0 || sys >= (int)e->sys.size()) return fail(e, OG_ERR_INVALID, "bad system id");
    HostSystem &h = e->sys[sys];
    const int n = h.d.n_atoms;
    if (interval < 0 || n_group < 0 || (n_group > 0 && !group_atoms))
        return fail(e, OG_ERR_INVALID, "negative interval or group size, or no group array");
    h.tr_interval = interval;
    h.tr_group.clear();
    if (interval == 0) return OG_OK;
    if (n_group == 0) {
        for (int a = 0; a < n; a++) h.tr_group.push_back(a);
    } else {
        for (int j = 0; j < n_group; j++) {
            if (group_atoms[j] < 0 || group_atoms[j] >= n) {
                h.tr_interval = 0;
                h.tr_group.clear();
                return fail(e, OG_ERR_INVALID, "trajectory group atom %d out of range", group_atoms[j]);
            }
            h.tr_group.push_back(group_atoms[j]);
        }
    }
    return OG_OK;
}

og_status og_take_frames(og_engine *e, int32_t sys, int32_t max, int64_t *step, float *crd, double *energies,
                         int32_t *n) {
    if (!e || !e->finalized) return fail(e, OG_ERR_STATE, "og_take_frames before og_finalize");
    if (sys < 0 || sys >= e->n_sys || max < 0 || !n || (max > 0 && (!step || !crd)))
        return fail(e, OG_ERR_INVALID, "bad system id or output arrays");
    const int m = e->sys[sys].dev.tr_slot;
    if (m < 0) return fail(e, OG_ERR_INVALID, "system %d has no trajectory output", sys);
    og_status s = logs_drain(e);
    if (s) return s;
    TrLog &T = e->tr[m];
    const size_t fc = 3 * (size_t)e->sys[sys].dev.tr_n;
    const int32_t avail = (int32_t)(T.step.size() - T.head);
    if (max == 0) {
        *n = avail;
        return OG_OK;
    }
    const int32_t k = std::min(max, avail);
    for (int32_t i = 0; i < k; i++) step[i] = T.step[T.head + i];
    memcpy(crd, T.crd.data() + T.head * fc, sizeof(float) * fc * k);
    if (energies) memcpy(energies, T.ene.data() + T.head * OG_N_ENERGY, sizeof(double) * OG_N_ENERGY * k);
    T.head += (size_t)k;
    if (T.head == T.step.size()) {
        T.step.clear();
        T.crd.clear();
        T.ene.clear();
        T.head = 0;
    }
    *n = k;
    return OG_OK;
}

// Per-step timing of the pair kernel (CUDA events on the engine's stream).  Not in the public
// header's main list: enabled by the benchmark.
og_status og_set_timing(og_engine *e, int32_t on) {
    if (!e) return OG_ERR_INVALID;
    e->timing = on == 2 ? 2 : (on != 0 ? 1 : 0);
    return OG_OK;
}

}  // extern "C"

extern "C" og_status og_get_flags(og_engine *e, int32_t *flags) {
    if (!e || !e->finalized || !flags) return OG_ERR_INVALID;
    int c[OG_CNT_SIZE];
    og_status s = read_counters(e, c);
    if (s) return s;
    *flags = c[OG_CNT_FLAGS];
    return OG_OK;
}

extern "C" og_status og_put_state(og_engine *e, int32_t sys, const double *crd, const double *vel_next) {
    if (!e || !e->finalized) return fail(e, OG_ERR_STATE, "og_put_state before og_finalize");
    if (sys < 0 || sys >= e->n_sys) return fail(e, OG_ERR_INVALID, "bad system id");
    const SysDev &D = e->sys[sys].dev;
    if (!e->d_stage) {
        og_status s = dalloc(e, &e->d_stage, 6 * (size_t)e->n_atoms);
        if (s) return s;
    }
    double *sc = e->d_stage, *sv = e->d_stage + 3 * (size_t)e->n_atoms;
    if (crd) CK(cudaMemcpyAsync(sc, crd, sizeof(double) * 3 * D.n_atoms, cudaMemcpyHostToDevice, e->stream));
    if (vel_next) CK(cudaMemcpyAsync(sv, vel_next, sizeof(double) * 3 * D.n_atoms, cudaMemcpyHostToDevice, e->stream));
    k_put_state<<<blocks(D.n_atoms, 256), 256, 0, e->stream>>>(D.n_atoms, D.atom_base, e->d_atom_sys, e->d_sys,
                                                                crd ? sc : nullptr, vel_next ? sv : nullptr, e->d_crd,
                                                                e->d_vel_next, e->d_atom_slot, e->d_slot_crd,
                                                                e->d_cell_origin, e->d_xq, e->d_xq_ref,
                                                                e->jl_skin * e->jl_skin, e->d_jl_stale,
                                                                e->d_xq_build, e->d_counters);
    LAUNCH_CHECK();
    return OG_OK;
}

extern "C" og_status og_get_state_async(og_engine *e, int32_t sys, double *crd, double *vel_next, double *energies) {
    if (!e || !e->finalized) return fail(e, OG_ERR_STATE, "og_get_state_async before og_finalize");
    if (sys < 0 || sys >= e->n_sys) return fail(e, OG_ERR_INVALID, "bad system id");
    const SysDev &D = e->sys[sys].dev;
    if (crd)
        CK(cudaMemcpyAsync(crd, e->d_crd + 3 * (size_t)D.atom_base, sizeof(double) * 3 * D.n_atoms,
                           cudaMemcpyDeviceToHost, e->stream));
    if (vel_next)
        CK(cudaMemcpyAsync(vel_next, e->d_vel_next + 3 * (size_t)D.atom_base, sizeof(double) * 3 * D.n_atoms,
                           cudaMemcpyDeviceToHost, e->stream));
    if (energies)
        CK(cudaMemcpyAsync(energies, e->d_energies + OG_N_ENERGY * (size_t)sys, sizeof(double) * OG_N_ENERGY,
                           cudaMemcpyDeviceToHost, e->stream));
    return OG_OK;
}

extern "C" og_status og_get_footprint(og_engine *e, int64_t *bytes_held, int64_t *bytes_peak) {
    if (!e) return OG_ERR_INVALID;
    if (bytes_held) *bytes_held = (int64_t)e->bytes_held;
    if (bytes_peak) *bytes_peak = (int64_t)e->bytes_peak;
    return OG_OK;
}

extern "C" og_status og_set_list_policy(og_engine *e, int32_t policy) {
    if (!e) return OG_ERR_INVALID;
    if (e->finalized) return fail(e, OG_ERR_STATE, "og_set_list_policy after og_finalize");
    if (policy != OG_LIST_FIXED && policy != OG_LIST_DISPLACEMENT)
        return fail(e, OG_ERR_INVALID, "list policy must be OG_LIST_FIXED or OG_LIST_DISPLACEMENT");
    e->list_policy = policy;
    return OG_OK;
}

extern "C" og_status og_get_list_builds(og_engine *e, int64_t *n_builds) {
    if (!e || !e->finalized || !n_builds) return OG_ERR_INVALID;
    int c[OG_CNT_SIZE];
    og_status s = read_counters(e, c);
    if (s) return s;
    *n_builds = c[OG_CNT_LIST_BUILDS];
    return OG_OK;
}

extern "C" og_status og_get_jlist_builds(og_engine *e, int64_t *n_builds) {
    if (!e || !e->finalized || !n_builds) return OG_ERR_INVALID;
    int c[OG_CNT_SIZE];
    og_status s = read_counters(e, c);
    if (s) return s;
    *n_builds = c[OG_CNT_JL_BUILDS];
    return OG_OK;
}

extern "C" og_status og_synchronize(og_engine *e) {
    if (!e) return OG_ERR_INVALID;
    CK(cudaStreamSynchronize(e->stream));
    return OG_OK;
}

extern "C" og_status og_step_async(og_engine *e, int32_t n_steps) {
    // og_step without the end-of-call flag check and without the capacity retry: the caller
    // checks og_get_flags at its own sync points
    if (!e || !e->finalized) return fail(e, OG_ERR_STATE, "og_step_async before og_finalize");
    for (int i = 0; i < n_steps; i++) {
        og_status s = logs_reserve(e, 1);  // synchronises only when a V-McMD log ring is full
        if (s) return s;
        // the call's last step (the one with energies) replays a one-step graph when nothing of
        // the step is decided on the host: the displacement policy's rebuilds are conditional
        // nodes; V-McMD systems keep the kernel-by-kernel path
        if (i == n_steps - 1 && e->use_graphs && !e->graph1_failed && e->timing != 1 &&
            e->list_policy == OG_LIST_DISPLACEMENT && e->n_vm == 0) {
            if (!e->graph1_exec && (s = capture_one_step(e))) return s;
            if (e->graph1_exec) {
                CK(cudaGraphLaunch(e->graph1_exec, e->stream));
                e->launches += e->graph1_kernels;
                e->graph_replays++;
                e->host_step++;
                continue;
            }
        }
        s = run_step(e, i == n_steps - 1);
        if (s) return s;
    }
    return OG_OK;
}

extern "C" og_status og_get_pair_count(og_engine *e, int32_t sys, int64_t *n_pairs) {
    if (!e || !e->finalized || !n_pairs) return OG_ERR_INVALID;
    if (sys < 0 || sys >= e->n_sys) return fail(e, OG_ERR_INVALID, "bad system id");
    double v = 0;
    CK(cudaMemcpy(&v, e->d_sys_acc + OG_ACC_SIZE * sys + OG_ACC_PAIRS, sizeof(double), cudaMemcpyDeviceToHost));
    *n_pairs = (int64_t)v;
    return OG_OK;
}

extern "C" og_status og_get_tuning(og_engine *e, int32_t *pair_variant, double *variant_ms) {
    if (!e) return OG_ERR_INVALID;
    if (pair_variant) *pair_variant = e->pair_variant;
    if (variant_ms)
        for (int v = 0; v < OG_N_PAIR_VARIANTS; v++) variant_ms[v] = e->variant_ms[v];
    return OG_OK;
}

// Fixed-order FP64 sum of value[i*stride] over each segment [seg_base[s], seg_base[s+1]) of a
// device array: the engine's two-level reduction (k_part / k_part_final), exposed for callers
// that keep per-item quantities on the device.  The partial sums live in a stream-ordered
// allocation released before return; the result does not depend on how segments are batched.
extern "C" og_status og_segment_sum(const double *d_values, int32_t stride, const int32_t *d_seg_base, int32_t n_seg,
                                    int32_t max_seg_len, double *d_out, void *cuda_stream) {
    if (!d_values || !d_seg_base || !d_out || n_seg <= 0 || stride <= 0 || max_seg_len < 0) return OG_ERR_INVALID;
    if (n_seg > OG_SEGMENT_SUM_MAX_SEGMENTS) return OG_ERR_CAPACITY;  // one grid row per segment
    if (cudaPeekAtLastError() != cudaSuccess) return OG_ERR_CUDA;     // the caller's error, left pending
    cudaStream_t st = (cudaStream_t)cuda_stream;
    const int max_chunks = (int)std::max(1LL, ((long long)max_seg_len + 4095) / 4096);
    double *part = nullptr;
    if (cudaMallocAsync((void **)&part, sizeof(double) * (size_t)n_seg * max_chunks, st) != cudaSuccess)
        return OG_ERR_NOMEM;
    dim3 grid(max_chunks, n_seg);
    k_part<1><<<grid, 256, 0, st>>>(d_values, stride, 0, d_seg_base, max_chunks, part);
    k_part_final<1><<<n_seg, 256, 0, st>>>(part, max_chunks, d_out, 1, 0, nullptr, 0);
    cudaError_t r = cudaGetLastError();
    cudaFreeAsync(part, st);
    return r == cudaSuccess ? OG_OK : OG_ERR_CUDA;
}

extern "C" og_status og_set_tuning(og_engine *e, int32_t pair_variant) {
    if (!e) return OG_ERR_INVALID;
    if (e->finalized) return fail(e, OG_ERR_STATE, "og_set_tuning after og_finalize");
    if (pair_variant < -1 || (pair_variant >= OG_N_PAIR_VARIANTS && pair_variant != OG_PAIR_VARIANT_F64))
        return fail(e, OG_ERR_INVALID, "pair variant must be -1, 0..%d or %d (FP64)", OG_N_PAIR_VARIANTS - 1,
                    OG_PAIR_VARIANT_F64);
    e->fixed_variant = pair_variant;
    return OG_OK;
}

extern "C" og_status og_set_graphs(og_engine *e, int32_t on) {
    if (!e) return OG_ERR_INVALID;
    e->use_graphs = on != 0;
    if (!e->use_graphs) drop_graph(e);
    e->graph_note.clear();
    return OG_OK;
}

extern "C" og_status og_get_graph_info(og_engine *e, int32_t *enabled, int64_t *replays, int64_t *kernels_per_replay,
                                       char *note) {
    if (!e) return OG_ERR_INVALID;
    if (enabled) *enabled = e->use_graphs ? 1 : 0;
    if (replays) *replays = e->graph_replays;
    if (kernels_per_replay) *kernels_per_replay = e->graph_kernels;
    if (note) snprintf(note, 256, "%s", e->graph_note.c_str());
    return OG_OK;
}

extern "C" og_status og_release_pool_memory(int32_t device) {
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        if (device < 0 || device >= 256) return OG_ERR_INVALID;
        pool = g_pool[device];
    }
    if (!pool) return OG_OK;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) return OG_ERR_CUDA;
    cudaError_t r = cudaDeviceSynchronize();
    if (r == cudaSuccess) r = cudaMemPoolTrimTo(pool, 0);
    cudaSetDevice(prev);
    return r == cudaSuccess ? OG_OK : OG_ERR_CUDA;
}

extern "C" og_status og_get_system_faults(og_engine *e, int32_t *faults) {
    if (!e || !e->finalized || !faults) return OG_ERR_INVALID;
    for (int k = 0; k < e->n_sys; k++) faults[k] = k < (int)e->faults.size() ? e->faults[k] : 0;
    return OG_OK;
}
