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
    size_t bytes = 0;
};

struct GraphEntry {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

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
    std::map<std::pair<int, cudaStream_t>, GraphEntry> graphs;
};

void set_error(const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);

int pattern_build(int n, const int* Ap, const int* Ai, const double* Ax, const int* q,
                  PatternObj** out);
void pattern_free(PatternObj* P);

void make_plan(const std::vector<PatternObj*>& pats, int block, int ctas_per_sm, int m, int vsize,
               SmemPlan& plan);
int batch_build(int nsys, PatternObj* const* pats, const lusp_batch_opts* o, BatchObj** out);
void batch_free(BatchObj* B);
int batch_launch(BatchObj* B, int what, cudaStream_t st);

}  // namespace lusp

// The opaque C handles (incomplete types in the public header) are these
// host objects; the C-ABI converts with reinterpret_cast.
