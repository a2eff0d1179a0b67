// Host-side context (the C ABI's opaque simp_ctx): one batch of resident
// basins ("instances").  A single-basin context is a batch of one.
#pragma once

#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "common.cuh"

// Host bookkeeping of one instance slot.
struct InstHost {
    bool active = false;
    bool retired = false;          // removed, storage kept until the next compaction
    simp::Inst I{};                // host copy of the device table entry
    int n = 0, nb = 0;             // particles and wall particles
    int id_base = 0;               // global particle id = id_base + local index
    double grid_hmax = 0.0;        // max(hsml) its grid was sized for
    long long order = 0;           // admission sequence: instances lie in this order in memory
    long long steps_since_sort = 0;
    long long steps_done = 0;
    std::vector<double> xb, massb; // its walls (re-binned when the layout changes)
    std::vector<double> bn;        // their normals b_normal(2, nb) (bf_Wang), empty until set
    // its walls in cell order: local cell keys and wall indices, for the
    // grid (cs, x0, y0) they were binned on
    std::vector<int> wall_key, wall_order;
    double wall_grid_cs = 0.0, wall_grid_x0 = 0.0, wall_grid_y0 = 0.0;
};

// Extents of a basin staged for admission, reduced on the device.
struct Extents {
    int n;
    double xmin, xmax, ymin, ymax, hmin, hmax;
    bool finite;
};

struct simp_ctx {
    simp_params prm{};
    simp::Phys phys{};
    int maxn = 0, maxnb = 0;       // capacities over all instances
    int max_inst = 1;
    int n = 0, nb = 0;             // particles and walls over all instances
    bool have_state = false;
    bool keep_diag = false;
    std::string err;
    cudaStream_t stream = nullptr;
    int device = 0;
    // single-basin contexts: get_state after steps enqueued without outputs
    // reads the fields no step writes (mass without mass evolution, hsml
    // when fixed) on a side stream while those steps run
    cudaStream_t side = nullptr;
    cudaEvent_t ev_graph = nullptr;   // recorded before each step graph launch
    cudaEvent_t ev_up[6] = {};        // a continued set_state's upload groups, and its start
    double *early_stage = nullptr;    // 2 maxn: those fields in the caller's order

    // instances
    std::vector<InstHost> insts;   // max_inst slots
    simp::Inst *inst_dev = nullptr;
    int ninst = 0;                 // table entries in use (highest active slot + 1)
    int id_stride = 0;             // 0 for a single basin, 1 << 21 for batches
    long long next_order = 0;      // admission counter
    // batches defer the layout and the sort of admissions and the removal of
    // retired basins to the next flush (abi.cu: flush_batch): the first
    // position written since, the admitted slots still to sort, and the
    // particles of retired basins still in place
    int pending_from = 0x7fffffff;
    std::vector<unsigned long long> pending_due;
    long long zombie_n = 0;
    int total_cells = 0;           // cell keys over all instances

    // particle state sets (device, cell order)
    simp::State s0{}, s1{};
    double *mass1 = nullptr;       // half-step mass when the mass update is on
    double *drhodt = nullptr;      // Benz hsml without con_density: the reference's drhodt, kept across steps
    double *k0 = nullptr;          // summation density in the step: the reference's kernel_zero, kept likewise
    double *red_dev = nullptr;     // per-block extents of a basin being admitted
    double *red_host = nullptr;    // (pinned copy)
    double *xr = nullptr, *yr = nullptr;  // sort positions (updated when the instance is re-sorted)
    double *xl = nullptr, *yl = nullptr;  // positions where each Verlet list was built
    int *cell = nullptr;           // sort-time cell key per particle
    int *id = nullptr;             // global particle id
    int *pinst = nullptr;          // instance slot of each particle (-1: being removed)
    // per-RHS intermediates from the kinematic pass
    double *tau11 = nullptr, *tau12 = nullptr, *tau22 = nullptr, *div = nullptr;
    // the stress pass's packed neighbour records (written by the kinematic pass)
    double2 *tau_a = nullptr, *tau_b = nullptr;   // plain form: (tau11, tau12), (tau22, m)
    float4 *tau_q = nullptr;                      // mixed form: (tau11, tau12, tau22, m)
    int *nbr = nullptr;            // kMaxNbr * maxn neighbour indices (column-major)
    int *nbr_count = nullptr;      // maxn
    int *nbr_tmp = nullptr;        // kMaxNbr * maxn: lists being renamed by a sort
    bool lists_valid = false;      // every particle's list was built by a kinematic pass
    bool pending_check = false;    // steps simp_gpu_step enqueued without outputs, status not read yet
    int *pair_j = nullptr;         // kMaxPairs * maxn exact pairs of the current RHS
    int *pair_count = nullptr;     // maxn
    void *pair_dw = nullptr;       // kernel gradient per pair: kDwRows x maxn float2 (mixed form only)
    // diagnostics (epsilon_11.. sigma_22, zeta, eta, p)
    double *diag = nullptr;        // 9 * maxn
    // rates of the last single_step (cell order): ax, ay, dhdt, dAdt
    double *rates = nullptr;       // 4 * maxn
    // regularisation terms of the current right-hand side (4 * maxn, only
    // with XSPH or artificial viscosity): viscous acceleration x, y and the
    // XSPH sum x, y (dx/dt after single_step)
    double *reg = nullptr;
    // wall particles, sorted by cell key
    double *bx = nullptr, *by = nullptr, *bm = nullptr;
    double *bnx = nullptr, *bny = nullptr;   // wall normals (bfa = 2 only)
    int *bid = nullptr;            // local wall index within its instance
    int *binst = nullptr;          // instance slot of each wall particle
    int *bcell = nullptr;          // cell key per wall slot
    int *bcell_start = nullptr;
    // cell lists
    int *cell_start = nullptr;
    size_t cell_cap = 0;
    // pair-pass implementation (SIMP_PASSES_*) and its tile shape
    int pass_impl = SIMP_PASSES_GATHER;
    int tile_threads = 256;        // particles per chunk = threads per block
    int tile_cap = 1024;           // halo particles a block stages
    // chunks of the tiled passes
    int total_rows = 0;            // cell rows over all instances
    int2 *row_map = nullptr;       // (instance, row) of each global row
    int *chunk_cnt = nullptr;      // chunks per row
    int *chunk_off = nullptr;      // their exclusive scan (+ total)
    simp::Chunk *chunks = nullptr;
    size_t row_cap = 0, chunk_cap = 0;
    // rebuild scratch
    int *cnt = nullptr;            // per-cell counters (cell_cap)
    int *perm = nullptr;           // maxn
    double *tmp = nullptr;         // 16 * max(maxn, maxnb) doubles reorder scratch
    int *itmp = nullptr;           // 5 * max(maxn, maxnb) ints
    void *scan_tmp = nullptr;
    size_t scan_tmp_bytes = 0;
    // scalars
    simp::Scalars *sc = nullptr;
    simp::Scalars *sc_host = nullptr;  // pinned mirror
    // NNPS export scratch
    int *pair_cnt = nullptr;       // maxn + 1
    int *bpair_cnt = nullptr;      // maxnb + 1
    int *pair_buf_i = nullptr, *pair_buf_j = nullptr;
    double *pair_buf_r = nullptr, *pair_buf_h = nullptr;
    size_t pair_buf_cap = 0;
    // step graph
    cudaGraphExec_t step_graph = nullptr;
    bool graph_stale = false;      // captured arguments changed since the last capture
    bool graph_diag = false;
    bool graph_profiled = false;
    long long graph_kernels = 0;   // kernels per replay
    // re-sort graph of a single basin: the kernels of one scheduled re-sort,
    // captured once and replayed while what they capture stays the same
    cudaGraphExec_t sort_graph = nullptr;
    struct SortKey {
        int n = -1, total_cells = -1;
        bool keep_lists = false;
        const void *cell_start = nullptr, *scan_tmp = nullptr;
        bool operator==(const SortKey &o) const {
            return n == o.n && total_cells == o.total_cells && keep_lists == o.keep_lists &&
                   cell_start == o.cell_start && scan_tmp == o.scan_tmp;
        }
    } sort_key;
    long long sort_kernels = 0;    // kernels per re-sort replay
    long long launches = 0;        // kernels launched by this context
    // per-kernel timing (events recorded inside the step graph)
    // (entry kProfKernels of prof_ms: the re-sorts between steps)
    static constexpr int kProfKernels = 5;
    bool profile = false;
    cudaEvent_t prof_ev[kProfKernels + 1] = {};
    cudaEvent_t sort_ev[2] = {};
    double prof_ms[kProfKernels + 1] = {};
    long long prof_steps = 0;
    long long rebuilds = 0;
};

namespace simp {

// Steps between the re-sorts of an instance into its cell grid.  A fixed
// schedule per instance (not a displacement test over the whole batch)
// keeps each instance's summation order independent of the other instances.
constexpr int kSortEvery = 16;
constexpr int kMaxSlots = 1024;

// cell_list.cu
struct DueMask {
    unsigned long long w[kMaxSlots / 64];
};
int rebuild(simp_ctx *c, const DueMask &due, int from, bool new_lists);   // sort into cell order
void launch_scan_i32(const int *in, int *out, int n, void *tmp, cudaStream_t s);
constexpr int kScanKernels = 4;         // kernels per launch_scan_i32
size_t scan_tmp_bytes(int n);

// passes.cu
// stress-pass epilogues: the rates (single_step), the predictor half step
// and the corrector (predictor_corrector), the Euler step, the leap-frog
// second half (time_integration.f90:86-148, 155-282, 289-391)
enum EpiMode : int { EPI_RATES = 0, EPI_PREDICT = 1, EPI_CORRECT = 2, EPI_EULER = 3, EPI_LEAP = 4 };
void launch_kinematic(simp_ctx *c, const State &s, bool diag);
void launch_stress(simp_ctx *c, const State &nb, const State &own, EpiMode mode);
// drho/dt over the last right-hand side's pairs with the updated velocities
// (con_density, Benz_hsml): rho_upd 0 none, 1 half step, 2 full step; tail:
// the step's final hsml, its bounds and the VP dt
void launch_density_rate(simp_ctx *c, const State &g, const State &v, int rho_upd, bool tail);
// summation density (den_alg 1) over the last right-hand side's pairs at
// state g: masses m_sum and densities rho_in of the reference's call, result
// into rho_out (v.rho, or scratch for launch_commit_rho); tail as above
void launch_sum_density(simp_ctx *c, const State &g, const State &v, const double *m_sum, const double *rho_in,
                        double *rho_out, bool tail);
void launch_commit_rho(simp_ctx *c, const double *src, const State &o);
void launch_step_finish(simp_ctx *c);
// XSPH and artificial viscosity of the right-hand side at s, over the pairs
// the kinematic pass just found (a no-op when both are off)
void launch_regularize(simp_ctx *c, const State &s);
void launch_copy_s1_to_s0(simp_ctx *c);
void launch_reset_stats(simp_ctx *c);

// tiled.cu
constexpr int kMinTileThreads = 64;
void build_chunks(simp_ctx *c);
int tiled_configure(simp_ctx *c);
size_t tiled_smem_bytes(int precision, int pass, int cap, int threads);

// abi.cu: device bytes per particle of capacity
double bytes_per_particle(const simp_params &p, bool single_basin = false);

// abi.cu: the step driver split for callers that overlap contexts
int step_enqueue(simp_ctx *c, int nsteps);
int step_complete(simp_ctx *c, double *current_time, double *dt);
// the status of steps enqueued without outputs (waits for them); SIMP_OK when none
int complete_pending(simp_ctx *c);
int batch_slot_state(simp_ctx *c, int slot, double *x, double *vx, double *mass, double *rho, double *hsml,
                     double *A, double *h, double *t);

// nnps_export.cu (instance 0 of the context)
int export_pairs(simp_ctx *c, int32_t *nip, int32_t *p_i, int32_t *p_j, double *r_ij,
                 double *hsml_ij, int32_t cap, int32_t *bnip, int32_t *bp_i, int32_t *bp_j,
                 double *br_ij, int32_t bcap);
int sum_density(simp_ctx *c, double *rho_out_dev);

}  // namespace simp

int simp_fail(simp_ctx *c, int code, const std::string &msg);
int simp_cuda_check(simp_ctx *c, cudaError_t e, const char *what);
#define SIMP_CUDA(c, expr)                                        \
    do {                                                          \
        cudaError_t _e = (expr);                                  \
        if (_e != cudaSuccess) return simp_cuda_check(c, _e, #expr); \
    } while (0)
