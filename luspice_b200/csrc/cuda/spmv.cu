// Whole-GPU sparse matrix-vector products.
//
//  - spmv.h (src/spmv.h:23-57): fp64 CSR with a group of 4 lanes per row
//    (circuit matrices average 3-8 entries per row), fp64 accumulation.
//  - lusp_sell_*: SELL-C-sigma with C in {8, 16, 32}: rows sorted by length
//    inside windows of sigma rows, slices of C rows stored column-major; one
//    warp per slice, 32/C lanes per row.  Values fp64, fp32, or fp16 after
//    Ruiz equilibration (range-checked at creation), int32 indices, fp64
//    accumulation.  Padding credits nothing: the algorithmic bytes are
//    nnz*(value+index) + row pointers + x + y.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "luspice_b200.h"
#include "spmv.h"
#include "engine_internal.h"

namespace {

constexpr int kCsrLanes = 4;

template <typename VT>
__global__ void __launch_bounds__(256)
csr_vector_kernel(int n, const int* __restrict__ rowptr, const int* __restrict__ colidx,
                  const VT* __restrict__ values, const double* __restrict__ x,
                  double* __restrict__ y) {
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) / kCsrLanes;
    const int sub = threadIdx.x % kCsrLanes;
    double acc = 0.0;
    if (g < n) {
        // Four independent partial sums keep four loads per lane in flight
        // (long rows would otherwise wait one memory latency per entry).
        const int p1 = rowptr[g + 1];
        double a1 = 0.0, a2 = 0.0, a3 = 0.0;
        int p = rowptr[g] + sub;
        for (; p + 3 * kCsrLanes < p1; p += 4 * kCsrLanes) {
            const int c0 = colidx[p], c1 = colidx[p + kCsrLanes], c2 = colidx[p + 2 * kCsrLanes],
                      c3 = colidx[p + 3 * kCsrLanes];
            acc = fma((double)values[p], __ldg(x + c0), acc);
            a1 = fma((double)values[p + kCsrLanes], __ldg(x + c1), a1);
            a2 = fma((double)values[p + 2 * kCsrLanes], __ldg(x + c2), a2);
            a3 = fma((double)values[p + 3 * kCsrLanes], __ldg(x + c3), a3);
        }
        for (; p < p1; p += kCsrLanes) acc = fma((double)values[p], __ldg(x + colidx[p]), acc);
        acc = (acc + a1) + (a2 + a3);
    }
#pragma unroll
    for (int o = kCsrLanes / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (g < n && sub == 0) y[g] = acc;
}

template <typename VT> __device__ __forceinline__ double ldv(const VT* p);
template <> __device__ __forceinline__ double ldv<double>(const double* p) { return __ldg(p); }
template <> __device__ __forceinline__ double ldv<float>(const float* p) { return (double)__ldg(p); }
template <> __device__ __forceinline__ double ldv<__half>(const __half* p) {
    return (double)__half2float(__ldg(p));
}

// Blocks [0, sell_blocks) take the slices; the blocks after them take the
// long rows, a warp per row (lanes over its entries, four partial sums per
// lane, a fixed-order warp reduction).
template <int C, typename VT>
__global__ void __launch_bounds__(256)
sell_kernel(int nslices, const int* __restrict__ ptr, const int* __restrict__ col,
            const VT* __restrict__ val, const int* __restrict__ perm,
            const double* __restrict__ x, double* __restrict__ y,
            const double* __restrict__ row_div, int sell_blocks, int nlong,
            const int* __restrict__ lrow, const int* __restrict__ lptr, const int* __restrict__ lcol,
            const VT* __restrict__ lval) {
    if ((int)blockIdx.x >= sell_blocks) {
        const int lane = threadIdx.x & 31;
        const int w = ((blockIdx.x - sell_blocks) * blockDim.x + threadIdx.x) >> 5;
        if (w >= nlong) return;
        const int p1 = lptr[w + 1];
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        int p = lptr[w] + lane;
        for (; p + 96 < p1; p += 128) {
            const int c0 = lcol[p], c1 = lcol[p + 32], c2 = lcol[p + 64], c3 = lcol[p + 96];
            a0 = fma(ldv<VT>(lval + p), __ldg(x + c0), a0);
            a1 = fma(ldv<VT>(lval + p + 32), __ldg(x + c1), a1);
            a2 = fma(ldv<VT>(lval + p + 64), __ldg(x + c2), a2);
            a3 = fma(ldv<VT>(lval + p + 96), __ldg(x + c3), a3);
        }
        for (; p < p1; p += 32) a0 = fma(ldv<VT>(lval + p), __ldg(x + lcol[p]), a0);
        double acc = (a0 + a1) + (a2 + a3);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            const int row = lrow[w];
            y[row] = row_div ? acc / row_div[row] : acc;
        }
        return;
    }
    constexpr int G = 32 / C;
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (s >= nslices) return;
    const int lane = threadIdx.x & 31;
    const int r = lane % C, sub = lane / C;
    const int base = ptr[s];
    const int L = (ptr[s + 1] - base) / C;
    double acc = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int t = sub;
    for (; t + 3 * G < L; t += 4 * G) {
        const int e = base + t * C + r, d = G * C;
        const int c0 = col[e], c1 = col[e + d], c2 = col[e + 2 * d], c3 = col[e + 3 * d];
        acc = fma(ldv<VT>(val + e), __ldg(x + c0), acc);
        a1 = fma(ldv<VT>(val + e + d), __ldg(x + c1), a1);
        a2 = fma(ldv<VT>(val + e + 2 * d), __ldg(x + c2), a2);
        a3 = fma(ldv<VT>(val + e + 3 * d), __ldg(x + c3), a3);
    }
    for (; t < L; t += G) {
        const int e = base + t * C + r;
        acc = fma(ldv<VT>(val + e), __ldg(x + col[e]), acc);
    }
    acc = (acc + a1) + (a2 + a3);
#pragma unroll
    for (int o = 16; o >= C; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (sub == 0) {
        const int row = perm[s * C + r];
        if (row >= 0) y[row] = row_div ? acc / row_div[row] : acc;
    }
}

// out = x / s elementwise (the column scaling undone on the input vector).
__global__ void unscale_kernel(int n, const double* __restrict__ x, const double* __restrict__ s,
                               double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = x[i] / s[i];
}

}  // namespace

struct SellObj {
    int n = 0, C = 32, sigma = 32, kind = 0, nslices = 0;
    long stored = 0, nnz = 0;
    int* d_ptr = nullptr;
    int* d_col = nullptr;
    void* d_val = nullptr;
    int* d_perm = nullptr;
    double* d_rs = nullptr;     // fp16: row scale
    double* d_cs = nullptr;     // fp16: column scale
    double* d_xs = nullptr;     // fp16: scaled x
    double smin = 0, smax = 0;
    // Rows much longer than the rest (supply nets) stay out of the slices
    // (one of them would set a whole slice's width): CSR, a warp per row.
    int nlong = 0;
    int* d_lrow = nullptr;      // [nlong] row
    int* d_lptr = nullptr;      // [nlong+1]
    int* d_lcol = nullptr;
    void* d_lval = nullptr;
};

// Ruiz equilibration (max norm): alternately scale rows and columns by
// 1/sqrt(max |a|) until every row and column maximum is within tol of 1.
// Same iteration as the reference's preprocessing (bench/test_lu_gpu_f32.cu:
// 249-269), written over CSR.
void lusp_ruiz_csr(int n, const int* rowptr, const int* colidx, const double* vals, int sweeps,
                   double tol, std::vector<double>& rs, std::vector<double>& cs) {
    rs.assign(n, 1.0);
    cs.assign(n, 1.0);
    std::vector<double> cmax(n);
    for (int it = 0; it < sweeps; it++) {
        double dev = 0.0;
        for (int i = 0; i < n; i++) {
            double m = 0.0;
            for (int p = rowptr[i]; p < rowptr[i + 1]; p++) m = std::max(m, std::fabs(vals[p]) * rs[i] * cs[colidx[p]]);
            if (m > 0) { rs[i] /= std::sqrt(m); dev = std::max(dev, std::fabs(1.0 - m)); }
        }
        std::fill(cmax.begin(), cmax.end(), 0.0);
        for (int i = 0; i < n; i++)
            for (int p = rowptr[i]; p < rowptr[i + 1]; p++)
                cmax[colidx[p]] = std::max(cmax[colidx[p]], std::fabs(vals[p]) * rs[i] * cs[colidx[p]]);
        for (int j = 0; j < n; j++)
            if (cmax[j] > 0) { cs[j] /= std::sqrt(cmax[j]); dev = std::max(dev, std::fabs(1.0 - cmax[j])); }
        if (dev < tol) break;
    }
}

extern "C" {

int csr_alloc_device(const CSRMatrix* A, int** d_rowptr, int** d_colidx, double** d_values) {
    if (!A || !d_rowptr || !d_colidx || !d_values || A->n <= 0) return 1;
    const size_t nr = ((size_t)A->n + 1) * sizeof(int);
    const size_t nc = (size_t)std::max<long long>(A->nnz, 1) * sizeof(int);
    const size_t nv = (size_t)std::max<long long>(A->nnz, 1) * sizeof(double);
    *d_rowptr = nullptr;
    *d_colidx = nullptr;
    *d_values = nullptr;
    if (cudaMalloc((void**)d_rowptr, nr) != cudaSuccess) return 1;
    if (cudaMalloc((void**)d_colidx, nc) != cudaSuccess) return 1;
    if (cudaMalloc((void**)d_values, nv) != cudaSuccess) return 1;
    if (cudaMemcpy(*d_rowptr, A->rowptr, nr, cudaMemcpyHostToDevice) != cudaSuccess) return 1;
    if (A->nnz > 0) {
        if (cudaMemcpy(*d_colidx, A->colidx, (size_t)A->nnz * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) return 1;
        if (cudaMemcpy(*d_values, A->values, (size_t)A->nnz * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) return 1;
    }
    return 0;
}

void spmv_launch(int n, const int* d_rowptr, const int* d_colidx, const double* d_values,
                 const double* d_x, double* d_y, void* stream) {
    if (n <= 0) return;
    const long threads = (long)n * kCsrLanes;
    const int grid = (int)((threads + 255) / 256);
    csr_vector_kernel<double><<<grid, 256, 0, (cudaStream_t)stream>>>(n, d_rowptr, d_colidx, d_values, d_x, d_y);
}

int lusp_csr_spmv32(int n, const int* d_rowptr, const int* d_colidx, const float* d_values,
                    const double* d_x, double* d_y, void* stream) {
    if (n <= 0 || !d_rowptr || !d_colidx || !d_values || !d_x || !d_y) return LUSP_EARG;
    const long threads = (long)n * kCsrLanes;
    const int grid = (int)((threads + 255) / 256);
    csr_vector_kernel<float><<<grid, 256, 0, (cudaStream_t)stream>>>(n, d_rowptr, d_colidx, d_values, d_x, d_y);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LUSP_OK : lusp::cuda_fail(e, "csr fp32 spmv launch");
}

int spmv_host(const CSRMatrix* A, const double* x, double* y, double* time_ms) {
    if (!A || !x || !y || A->n <= 0) return 1;
    int *dr = nullptr, *dc = nullptr;
    double *dv = nullptr, *dx = nullptr, *dy = nullptr;
    int rc = 1;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const size_t nb = (size_t)A->n * sizeof(double);
    do {
        if (csr_alloc_device(A, &dr, &dc, &dv)) break;
        if (cudaMalloc((void**)&dx, nb) != cudaSuccess) break;
        if (cudaMalloc((void**)&dy, nb) != cudaSuccess) break;
        if (cudaMemcpy(dx, x, nb, cudaMemcpyHostToDevice) != cudaSuccess) break;
        spmv_launch(A->n, dr, dc, dv, dx, dy, 0);
        if (cudaDeviceSynchronize() != cudaSuccess) break;
        if (time_ms) {
            cudaEventCreate(&e0);
            cudaEventCreate(&e1);
            cudaEventRecord(e0, 0);
            spmv_launch(A->n, dr, dc, dv, dx, dy, 0);
            cudaEventRecord(e1, 0);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            *time_ms = ms;
        }
        if (cudaGetLastError() != cudaSuccess) break;
        if (cudaMemcpy(y, dy, nb, cudaMemcpyDeviceToHost) != cudaSuccess) break;
        rc = 0;
    } while (0);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(dr);
    cudaFree(dc);
    cudaFree(dv);
    cudaFree(dx);
    cudaFree(dy);
    return rc;
}

int lusp_sell_create(int n, const int* rowptr, const int* colidx, const double* vals, int C,
                     int sigma, int value_kind, lusp_sell** out) {
    if (!out) return LUSP_EARG;
    *out = nullptr;
    if (n <= 0 || !rowptr || !colidx || !vals) return LUSP_EARG;
    if (C != 8 && C != 16 && C != 32) { lusp::set_error("sell_create: C must be 8, 16 or 32"); return LUSP_EARG; }
    if (value_kind < 0 || value_kind > 2) return LUSP_EARG;
    sigma = std::max(sigma, C);
    SellObj* S = nullptr;
    try {
        S = new SellObj();
        S->n = n;
        S->C = C;
        S->sigma = sigma;
        S->kind = value_kind;
        S->nnz = rowptr[n];
        std::vector<double> rs, cs;
        if (value_kind == 2) {
            lusp_ruiz_csr(n, rowptr, colidx, vals, 30, 1e-6, rs, cs);
            double mn = INFINITY, mx = 0.0;
            for (int i = 0; i < n; i++)
                for (int p = rowptr[i]; p < rowptr[i + 1]; p++) {
                    const double a = std::fabs(vals[p] * rs[i] * cs[colidx[p]]);
                    if (a == 0.0) continue;
                    mn = std::min(mn, a);
                    mx = std::max(mx, a);
                }
            S->smin = mn;
            S->smax = mx;
            // fp16 normal range: [2^-14, 65504].
            if (!(mn >= 6.103515625e-05) || !(mx <= 65504.0)) {
                lusp::set_error("sell_create: Ruiz-scaled values span [%.3e, %.3e], outside the fp16 normal range", mn, mx);
                delete S;
                return LUSP_EARG;
            }
        }
        std::vector<int> len(n), perm, lrows;
        for (int i = 0; i < n; i++) len[i] = rowptr[i + 1] - rowptr[i];
        // Rows longer than max(256, 8 x the mean row length) go to the long
        // list; the rest are sorted by length inside windows of sigma rows.
        const long thr = std::max<long>(256, 8 * ((rowptr[n] + n - 1) / n));
        for (int i = 0; i < n; i++) (len[i] > thr ? lrows : perm).push_back(i);
        const int nsh = (int)perm.size();
        for (int w0 = 0; w0 < nsh; w0 += sigma) {
            const int w1 = std::min(nsh, w0 + sigma);
            std::stable_sort(perm.begin() + w0, perm.begin() + w1, [&len](int a, int b) { return len[a] > len[b]; });
        }
        const int ns = (nsh + C - 1) / C;
        S->nslices = ns;
        std::vector<int> ptr(ns + 1, 0), hperm((size_t)ns * C, -1);
        for (int s = 0; s < ns; s++) {
            int ml = 0;
            for (int r = 0; r < C; r++) {
                const int k = s * C + r;
                if (k < nsh) { hperm[k] = perm[k]; ml = std::max(ml, len[perm[k]]); }
            }
            ptr[s + 1] = ptr[s] + ml * C;
        }
        const long total = ptr[ns];
        S->stored = total;
        std::vector<int> hcol(std::max<long>(total, 1), 0);
        std::vector<double> hval(std::max<long>(total, 1), 0.0);
        for (int s = 0; s < ns; s++)
            for (int r = 0; r < C; r++) {
                const int k = s * C + r;
                if (k >= nsh) continue;
                const int row = perm[k];
                const int L = (ptr[s + 1] - ptr[s]) / C;
                for (int t = 0; t < L; t++) {
                    const long e = ptr[s] + (long)t * C + r;
                    if (t < len[row]) {
                        const int p = rowptr[row] + t;
                        hcol[e] = colidx[p];
                        hval[e] = value_kind == 2 ? vals[p] * rs[row] * cs[colidx[p]] : vals[p];
                    } else {
                        hcol[e] = row < n ? row : 0;
                    }
                }
            }
        const size_t vsz = value_kind == 0 ? 8 : value_kind == 1 ? 4 : 2;
        cudaError_t e = cudaSuccess;
        e = cudaMalloc((void**)&S->d_ptr, (ns + 1) * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc((void**)&S->d_col, hcol.size() * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc(&S->d_val, hcol.size() * vsz);
        if (e == cudaSuccess) e = cudaMalloc((void**)&S->d_perm, hperm.size() * sizeof(int));
        if (e == cudaSuccess) e = cudaMemcpy(S->d_ptr, ptr.data(), (ns + 1) * sizeof(int), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(S->d_col, hcol.data(), hcol.size() * sizeof(int), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(S->d_perm, hperm.data(), hperm.size() * sizeof(int), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            if (value_kind == 0) {
                e = cudaMemcpy(S->d_val, hval.data(), hval.size() * 8, cudaMemcpyHostToDevice);
            } else if (value_kind == 1) {
                std::vector<float> f(hval.size());
                for (size_t t = 0; t < f.size(); t++) f[t] = (float)hval[t];
                e = cudaMemcpy(S->d_val, f.data(), f.size() * 4, cudaMemcpyHostToDevice);
            } else {
                std::vector<__half> h(hval.size());
                for (size_t t = 0; t < h.size(); t++) h[t] = __double2half(hval[t]);
                e = cudaMemcpy(S->d_val, h.data(), h.size() * 2, cudaMemcpyHostToDevice);
            }
        }
        // Long rows: CSR in their original order, values as stored above.
        S->nlong = (int)lrows.size();
        if (e == cudaSuccess && S->nlong > 0) {
            std::vector<int> lptr(S->nlong + 1, 0), lcol;
            std::vector<double> lv;
            for (int t = 0; t < S->nlong; t++) {
                const int row = lrows[t];
                for (int p = rowptr[row]; p < rowptr[row + 1]; p++) {
                    lcol.push_back(colidx[p]);
                    lv.push_back(value_kind == 2 ? vals[p] * rs[row] * cs[colidx[p]] : vals[p]);
                }
                lptr[t + 1] = (int)lcol.size();
            }
            S->stored += (long)lcol.size();
            e = cudaMalloc((void**)&S->d_lrow, lrows.size() * sizeof(int));
            if (e == cudaSuccess) e = cudaMalloc((void**)&S->d_lptr, lptr.size() * sizeof(int));
            if (e == cudaSuccess) e = cudaMalloc((void**)&S->d_lcol, lcol.size() * sizeof(int));
            if (e == cudaSuccess) e = cudaMalloc(&S->d_lval, lv.size() * vsz);
            if (e == cudaSuccess) e = cudaMemcpy(S->d_lrow, lrows.data(), lrows.size() * sizeof(int), cudaMemcpyHostToDevice);
            if (e == cudaSuccess) e = cudaMemcpy(S->d_lptr, lptr.data(), lptr.size() * sizeof(int), cudaMemcpyHostToDevice);
            if (e == cudaSuccess) e = cudaMemcpy(S->d_lcol, lcol.data(), lcol.size() * sizeof(int), cudaMemcpyHostToDevice);
            if (e == cudaSuccess) {
                if (value_kind == 0) {
                    e = cudaMemcpy(S->d_lval, lv.data(), lv.size() * 8, cudaMemcpyHostToDevice);
                } else if (value_kind == 1) {
                    std::vector<float> f(lv.size());
                    for (size_t t = 0; t < f.size(); t++) f[t] = (float)lv[t];
                    e = cudaMemcpy(S->d_lval, f.data(), f.size() * 4, cudaMemcpyHostToDevice);
                } else {
                    std::vector<__half> h(lv.size());
                    for (size_t t = 0; t < h.size(); t++) h[t] = __double2half(lv[t]);
                    e = cudaMemcpy(S->d_lval, h.data(), h.size() * 2, cudaMemcpyHostToDevice);
                }
            }
        }
        if (e == cudaSuccess && value_kind == 2) {
            e = cudaMalloc((void**)&S->d_rs, n * sizeof(double));
            if (e == cudaSuccess) e = cudaMalloc((void**)&S->d_cs, n * sizeof(double));
            if (e == cudaSuccess) e = cudaMalloc((void**)&S->d_xs, n * sizeof(double));
            if (e == cudaSuccess) e = cudaMemcpy(S->d_rs, rs.data(), n * sizeof(double), cudaMemcpyHostToDevice);
            if (e == cudaSuccess) e = cudaMemcpy(S->d_cs, cs.data(), n * sizeof(double), cudaMemcpyHostToDevice);
        }
        if (e != cudaSuccess) {
            lusp_sell_destroy(reinterpret_cast<lusp_sell*>(S));
            return lusp::cuda_fail(e, "sell_create");
        }
    } catch (const std::bad_alloc&) {
        delete S;
        return LUSP_EALLOC;
    }
    *out = reinterpret_cast<lusp_sell*>(S);
    return LUSP_OK;
}

void lusp_sell_destroy(lusp_sell* hs) {
    SellObj* S = reinterpret_cast<SellObj*>(hs);
    if (!S) return;
    cudaFree(S->d_ptr);
    cudaFree(S->d_col);
    cudaFree(S->d_val);
    cudaFree(S->d_perm);
    cudaFree(S->d_rs);
    cudaFree(S->d_cs);
    cudaFree(S->d_xs);
    cudaFree(S->d_lrow);
    cudaFree(S->d_lptr);
    cudaFree(S->d_lcol);
    cudaFree(S->d_lval);
    delete S;
}

int lusp_sell_spmv(const lusp_sell* hs, const double* d_x, double* d_y, void* stream) {
    const SellObj* S = reinterpret_cast<const SellObj*>(hs);
    if (!S || !d_x || !d_y) return LUSP_EARG;
    cudaStream_t st = (cudaStream_t)stream;
    const double* xin = d_x;
    if (S->kind == 2) {
        // A x = Dr^-1 (Dr A Dc) (Dc^-1 x): the stored values are Dr A Dc.
        unscale_kernel<<<(S->n + 255) / 256, 256, 0, st>>>(S->n, d_x, S->d_cs, S->d_xs);
        xin = S->d_xs;
    }
    const int sell_blocks = (int)(((long)S->nslices * 32 + 255) / 256);
    const int long_blocks = (int)(((long)S->nlong * 32 + 255) / 256);
    const int grid = sell_blocks + long_blocks;
    const double* rsc = S->kind == 2 ? S->d_rs : nullptr;
#define LUSP_SELL_CASE(CC)                                                                        \
    if (S->C == CC) {                                                                             \
        if (S->kind == 0)                                                                         \
            sell_kernel<CC, double><<<grid, 256, 0, st>>>(S->nslices, S->d_ptr, S->d_col,         \
                (const double*)S->d_val, S->d_perm, xin, d_y, rsc, sell_blocks, S->nlong,         \
                S->d_lrow, S->d_lptr, S->d_lcol, (const double*)S->d_lval);                       \
        else if (S->kind == 1)                                                                    \
            sell_kernel<CC, float><<<grid, 256, 0, st>>>(S->nslices, S->d_ptr, S->d_col,          \
                (const float*)S->d_val, S->d_perm, xin, d_y, rsc, sell_blocks, S->nlong,          \
                S->d_lrow, S->d_lptr, S->d_lcol, (const float*)S->d_lval);                        \
        else                                                                                      \
            sell_kernel<CC, __half><<<grid, 256, 0, st>>>(S->nslices, S->d_ptr, S->d_col,         \
                (const __half*)S->d_val, S->d_perm, xin, d_y, rsc, sell_blocks, S->nlong,         \
                S->d_lrow, S->d_lptr, S->d_lcol, (const __half*)S->d_lval);                       \
    }
    LUSP_SELL_CASE(8)
    LUSP_SELL_CASE(16)
    LUSP_SELL_CASE(32)
#undef LUSP_SELL_CASE
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LUSP_OK : lusp::cuda_fail(e, "sell spmv launch");
}

int lusp_sell_info(const lusp_sell* hs, long* stored, long* nnz, double* smin, double* smax) {
    const SellObj* S = reinterpret_cast<const SellObj*>(hs);
    if (!S) return LUSP_EARG;
    if (stored) *stored = S->stored;
    if (nnz) *nnz = S->nnz;
    if (smin) *smin = S->smin;
    if (smax) *smax = S->smax;
    return LUSP_OK;
}

}  // extern "C"
