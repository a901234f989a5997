// Host-side objects behind the opaque C-ABI handles.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <map>
#include <utility>
#include <vector>

#include "luspice_b200.h"
#include "../host/lusp_host.h"
#include "engine.cuh"

namespace lusp {

struct PatternObj {
    StaticPattern S;
    PatternDev desc{};               // host copy holding device pointers
    PatternDev* d_desc = nullptr;
    int* d_block = nullptr;
    void* d_rel = nullptr;           // relative update slots (rel_ptr, rel)
    size_t bytes = 0;
};

// Everything one persistent launch needs (device descriptors already
// uploaded).
struct LaunchArgs {
    const SysDev* d_sys = nullptr;
    int nsys = 0;
    int* d_queue = nullptr;
    SmemPlan plan{};
    SolveParams prm{};
    int prec = LUSP_MIXED;
    int inner = 0;
    int what = LUSP_RUN_BOTH;
    int ir64 = 0;                    // fp64 factors solved by GMRES-IR, not directly
    cudaEvent_t* kev = nullptr;      // per-kernel timing events of the main rung (or null)
    int block = 256;
    int grid = 1;
    SmemPlan rplan{};                // refactorization kernel
    int rblock = 1024;
    int rgrid = 1;
    int rcluster = 1;                // CTAs per system (thread-block cluster)
    SpreadArgs rspread{};            // CTAs per system in global-memory sync (group 0: off)
    SmemPlan dplan{};                // dense trailing-block kernel (dgrid 0: none)
    int dblock = 512;
    int dgrid = 0;
    int dcluster = 1;                // CTAs per system of the dense-block kernel (cluster)
    // Escalation ladder after a mixed solve (rungs: bit 0 P-safe, bit 1
    // P-hard; 0 none): fp64 kernels over the slots the solve kernel takes.
    int rungs = 0;
    EscDev esc{};
    SmemPlan xplan{}, xrplan{}, xdplan{};
    int xblock = 512, xgrid = 0, xrblock = 1024, xrgrid = 0, xrcluster = 1, xdblock = 512, xdgrid = 0;
    SpreadArgs xrspread{};           // always off for the ladder
    SolveParams xprm{};              // P-safe parameters; P-hard adds the shift
    double hard_shift = 1e-7;
};

// Queue words of one launch: three work counters per rung (P-fast, P-safe,
// P-hard) in words 0..8, then the ladder's control words from word 10: two
// slot counters and the 64-bit pool counter (words 12..13, 8-byte aligned
// because the queue block is).
constexpr int kQueueWords = 16;
constexpr int kLadderCtl = 10;
static_assert((kLadderCtl + 2) % 2 == 0 && kLadderCtl + 4 <= kQueueWords, "ladder control words");

struct GraphEntry {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

// Device memory and launch shapes of a ladder for up to cap systems of
// pats (fp64 plans, storage pool, spill, slot descriptors, P-hard list).
// pool: bytes of fp64 system storage (0: room for cap of the largest).
struct LadderPlan {
    size_t pool = 0, spill = 0, bytes = 0;
};
int ladder_setup(const std::vector<PatternObj*>& pats, const lusp_batch_opts& o, int cap, LaunchArgs& a,
                 LadderPlan& lp, size_t pool = 0);
// Points the ladder into mem (lp.bytes, 256-byte aligned); queue: the
// launch's queue words.
void ladder_bind(LaunchArgs& a, const LadderPlan& lp, char* mem, int* queue);

struct BatchObj {
    int nsys = 0;
    int prec = LUSP_MIXED;
    lusp_batch_opts opts{};
    std::vector<PatternObj*> pats;
    std::vector<SysDev> h_sys;
    SysDev* d_sys = nullptr;
    SysStats* d_stats = nullptr;
    int* d_queue = nullptr;
    char* d_block = nullptr;
    char* d_ladder = nullptr;        // escalation ladder storage (may be null)
    size_t bytes = 0;
    double* d_vals = nullptr;        // all systems' values, concatenated
    double* d_rhs = nullptr;         // all right-hand sides
    double* d_x = nullptr;           // all solutions
    std::vector<size_t> val_off, vec_off;
    SmemPlan plan{};
    SolveParams prm{};
    int block = 256;
    int grid = 1;
    int launches = 0;
    cudaEvent_t kev[4] = {nullptr, nullptr, nullptr, nullptr};   // per-kernel timing (lusp_batch_time_kernels)
    LaunchArgs launch{};
    std::map<std::pair<int, cudaStream_t>, GraphEntry> graphs;
};

void set_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);

// dense_tail: -1 cost model, 0 none, > 0 that many trailing columns.
int pattern_build(int n, const int* Ap, const int* Ai, const double* Ax, const int* q,
                  PatternObj** out, int dense_tail = -1);
void pattern_free(PatternObj* P);

void make_plan(const std::vector<PatternObj*>& pats, int block, int ctas_per_sm, int m, int vsize,
               SmemPlan& plan);
int batch_build(int nsys, PatternObj* const* pats, const lusp_batch_opts* o, BatchObj** out);

// Building blocks shared by batches and the serving loop.
int check_opts(const lusp_batch_opts* o);
void fill_params(SolveParams& prm, const lusp_batch_opts& o);
int plan_for(const std::vector<PatternObj*>& pats, const lusp_batch_opts& o, SmemPlan& plan);
int kernel_occupancy(int prec, int inner, size_t smem, int block, int* occ);
// spread: the spread-mode kernel (several CTAs per system, global-memory
// synchronization) instead of the cluster kernel.
int refactor_occupancy(int prec, size_t smem, int block, int* occ, bool spread = false);
int refactor_block(const lusp_batch_opts& o, int nsys);
// Solve-kernel CTA size and plan target for nsys systems when left at 0.
void resolve_solve_shape(lusp_batch_opts& o, int nsys);
// ctas_per_sm: CTAs sharing an SM's shared memory (0: 1024 / threads).
void make_refactor_plan(const std::vector<PatternObj*>& pats, int threads, int vsize, SmemPlan& plan,
                        int ctas_per_sm = 0);
// Refactorization kernel block, plan and grid for nsys systems of pats.
int refactor_setup(const std::vector<PatternObj*>& pats, const lusp_batch_opts& o, int nsys, LaunchArgs& a);
// Kernels one launch with these RUN_* flags issues.
int launch_kernel_count(const LaunchArgs& a, int what);
void make_dense_plan(const std::vector<PatternObj*>& pats, int threads, SmemPlan& plan);
size_t system_private_bytes(const StaticPattern& S, size_t vs, int m);
int tail_ld(const StaticPattern& S);

char* carve_system(SysDev& D, char* p, const StaticPattern& S, size_t vs, int m);
size_t spill_bytes(int grid, int block, int colmax, const SmemPlan& rplan);
int launch_systems(const LaunchArgs& a, cudaStream_t st);
// Completes the merged slot array of one system (U part, diagonal, dense
// block) on stream st.
int batch_merge_factor(BatchObj* B, int sys, cudaStream_t st);
int sm_count();
// Loads every engine kernel into the current context now (not lazily at
// its first launch).
int preload_kernels();
void batch_free(BatchObj* B);
// timed: record the per-kernel timing events when the batch has them (not
// in graph capture).
int batch_launch(BatchObj* B, int what, cudaStream_t st, bool timed = false);

}  // namespace lusp

// The opaque C handles (incomplete types in the public header) are these
// host objects; the C-ABI converts with reinterpret_cast.
