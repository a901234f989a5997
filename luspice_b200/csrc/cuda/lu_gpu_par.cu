// Single-block sparse LU with partial pivoting decided on the device, and
// its triangular solve: the kernels declared by lu_gpu_par.h.
//
// lu_factor_par_kernel: one CTA of 256 threads walks the columns in order.
// For column k the dense work vector x lives in shared memory (n doubles);
// the columns j < k that update it are discovered as a bitmap over pivot
// positions: A(:,k) seeds the bits of its pivoted rows, and every column
// applied sets the bits of the pivoted rows it touches (always at positions
// above the current one).  Warp 0 finds the lowest set bit with ballots, so
// the updates are applied in ascending pivot order, exactly the order of
// the single-thread reference kernel (src/lu_gpu.cu:64-77); exact zeros skip
// their column as there.  Pivot search, U and L extraction are block-wide
// ordered compactions over the row index, giving the same entry order as the
// single-thread kernel.  Multiply and subtract are separately rounded.
#include <cuda_runtime.h>

#include "lu_gpu_par.h"

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

// Exclusive block scan of 0/1 flags in thread order; returns the prefix and
// writes the total to *total (all threads).
__device__ __forceinline__ int block_flag_scan(bool flag, int* wsum, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned b = __ballot_sync(0xffffffffu, flag);
    const int before = __popc(b & ((1u << lane) - 1u));
    __syncthreads();
    if (lane == 0) wsum[warp] = __popc(b);
    __syncthreads();
    int off = 0, tot = 0;
    for (int w = 0; w < kWarps; w++) {
        const int c = wsum[w];
        if (w < warp) off += c;
        tot += c;
    }
    *total = tot;
    return off + before;
}

}  // namespace

__global__ void __launch_bounds__(256)
lu_factor_par_kernel(int n, const int* Ap, const int* Ai, const double* Ax, const int* diagrow,
                     int* Lp, int* Li, double* Lx, long Lcap, int* Up, int* Ui, double* Ux,
                     long Ucap, int* pinv, int* xi, double* xg, int* lnnz, int* unnz,
                     int* singular_out) {
    (void)xg;
    if (blockDim.x != kThreads) {
        if (threadIdx.x == 0) *singular_out = -3;
        return;
    }
    extern __shared__ __align__(16) unsigned char lupar_smem[];
    double* x = (double*)lupar_smem;                       // [n]
    unsigned* cand = (unsigned*)(x + n);                    // [ceil(n/32)] within the 4n region
    __shared__ int wsum[kWarps];
    __shared__ double red_v[kWarps];
    __shared__ int red_i[kWarps];
    __shared__ int s_j, s_ipiv, s_status;
    __shared__ double s_pivot;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nwords = (n + 31) >> 5;
    int* rowat = xi;

    for (int i = tid; i < n; i += kThreads) {
        x[i] = 0.0;
        pinv[i] = -1;
        rowat[i] = -1;
    }
    for (int w = tid; w < nwords; w += kThreads) cand[w] = 0u;
    if (tid == 0) s_status = -1;
    __syncthreads();

    long lnz = 0, unz = 0;
    for (int k = 0; k < n; k++) {
        if (tid == 0) {
            Lp[k] = (int)lnz;
            Up[k] = (int)unz;
        }
        // 1. x = A(:,k) (assignment, the last duplicate wins) and seeds.
        const int a0 = Ap[k], a1 = Ap[k + 1];
        for (int p = a0 + tid; p < a1; p += kThreads) {
            const int i = Ai[p];
            bool last = true;
            for (int p2 = p + 1; p2 < a1; p2++)
                if (Ai[p2] == i) { last = false; break; }
            if (last) x[i] = Ax[p];
            const int J = pinv[i];
            if (J >= 0) atomicOr(&cand[J >> 5], 1u << (J & 31));
        }
        __syncthreads();
        // 2. Left-looking updates in ascending pivot position.
        int cur = 0;
        while (true) {
            if (warp == 0) {
                int found = -1;
                for (int w0 = cur >> 5; w0 < nwords && found < 0; w0 += 32) {
                    const int w = w0 + lane;
                    unsigned bits = (w < nwords) ? cand[w] : 0u;
                    if (w == (cur >> 5)) bits &= ~((1u << (cur & 31)) - 1u);
                    const unsigned any = __ballot_sync(0xffffffffu, bits != 0u);
                    if (any) {
                        const int src = __ffs(any) - 1;
                        const unsigned wb = __shfl_sync(0xffffffffu, bits, src);
                        found = ((w0 + src) << 5) + (__ffs(wb) - 1);
                    }
                }
                if (lane == 0) {
                    s_j = found;
                    if (found >= 0) cand[found >> 5] &= ~(1u << (found & 31));
                }
            }
            __syncthreads();
            const int j = s_j;
            if (j < 0) break;
            const double xr = x[rowat[j]];
            if (xr != 0.0) {
                for (int p = Lp[j] + 1 + tid; p < Lp[j + 1]; p += kThreads) {
                    const int i = Li[p];
                    x[i] = __dsub_rn(x[i], __dmul_rn(Lx[p], xr));
                    const int J = pinv[i];
                    if (J >= 0) atomicOr(&cand[J >> 5], 1u << (J & 31));
                }
            }
            cur = j + 1;
            __syncthreads();
        }
        // 3. Pivot search (largest |x|, smallest row on ties) and U(:,k).
        double bv = -1.0;
        int bi = -1;
        for (int base = 0; base < n; base += kThreads) {
            const int i = base + tid;
            bool isU = false;
            double xi_v = 0.0;
            int pi = -1;
            if (i < n) {
                pi = pinv[i];
                xi_v = x[i];
                if (pi < 0) {
                    const double t = fabs(xi_v);
                    if (t > bv) { bv = t; bi = i; }
                } else {
                    isU = xi_v != 0.0;
                }
            }
            int tot;
            const int off = block_flag_scan(isU, wsum, &tot);
            if (unz + tot > Ucap) {
                if (tid == 0) s_status = -2;
            } else if (isU) {
                Ui[unz + off] = pi;
                Ux[unz + off] = xi_v;
            }
            unz += tot;
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double v2 = __shfl_down_sync(0xffffffffu, bv, o);
            const int i2 = __shfl_down_sync(0xffffffffu, bi, o);
            if (v2 > bv || (v2 == bv && i2 >= 0 && (bi < 0 || i2 < bi))) { bv = v2; bi = i2; }
        }
        if (lane == 0) { red_v[warp] = bv; red_i[warp] = bi; }
        __syncthreads();
        if (tid == 0) {
            double a = -1.0;
            int ip = -1;
            for (int w = 0; w < kWarps; w++) {
                const double v2 = red_v[w];
                const int i2 = red_i[w];
                if (v2 > a || (v2 == a && i2 >= 0 && (ip < 0 || i2 < ip))) { a = v2; ip = i2; }
            }
            if (s_status == -1) {
                if (ip == -1 || a <= 0.0) {
                    s_status = k;
                } else {
                    const int ck = diagrow[k];
                    if (pinv[ck] < 0 && fabs(x[ck]) >= a) ip = ck;
                    s_ipiv = ip;
                    s_pivot = x[ip];
                    if (unz + 1 > Ucap || lnz + 1 > Lcap) {
                        s_status = -2;
                    } else {
                        Ui[unz] = k;
                        Ux[unz] = s_pivot;
                        pinv[ip] = k;
                        rowat[k] = ip;
                        Li[lnz] = ip;
                        Lx[lnz] = 1.0;
                    }
                }
            }
        }
        __syncthreads();
        if (s_status != -1) {
            if (tid == 0) *singular_out = s_status;
            return;
        }
        unz += 1;
        lnz += 1;
        // 4. L(:,k): unpivoted nonzero rows ascending, scaled by the pivot;
        //    the work vector is cleared on the way.
        const double pivot = s_pivot;
        for (int base = 0; base < n; base += kThreads) {
            const int i = base + tid;
            bool isL = false;
            double v = 0.0;
            if (i < n) {
                v = x[i];
                isL = pinv[i] < 0 && v != 0.0;
                x[i] = 0.0;
            }
            int tot;
            const int off = block_flag_scan(isL, wsum, &tot);
            if (lnz + tot > Lcap) {
                if (tid == 0) s_status = -2;
            } else if (isL) {
                Li[lnz + off] = i;
                Lx[lnz + off] = __ddiv_rn(v, pivot);
            }
            lnz += tot;
        }
        __syncthreads();
        if (s_status != -1) {
            if (tid == 0) *singular_out = s_status;
            return;
        }
    }
    if (tid == 0) {
        Lp[n] = (int)lnz;
        Up[n] = (int)unz;
    }
    for (long p = tid; p < lnz; p += kThreads) Li[p] = pinv[Li[p]];
    __syncthreads();
    if (tid == 0) {
        *lnnz = (int)lnz;
        *unnz = (int)unz;
        *singular_out = -1;
    }
}

// pb = P b; L y = pb by columns (unit diagonal first); U z = y by columns
// (diagonal last); x = Q z.  Same operation sequence as splu.h:210-239, so
// the result is bitwise that of the host solve on the same factors.
__global__ void __launch_bounds__(256)
trisolve_par_kernel(int n, const int* Lp, const int* Li, const double* Lx, const int* Up,
                    const int* Ui, const double* Ux, const int* pinv, const int* q,
                    const double* b, double* x, int* work_i, double* work_d) {
    const int tid = threadIdx.x, nt = blockDim.x;
    int* rowat = work_i;
    double* pb = work_d;
    double* y = work_d + n;
    for (int i = tid; i < n; i += nt) rowat[i] = -1;
    __syncthreads();
    for (int i = tid; i < n; i += nt)
        if (pinv[i] >= 0) rowat[pinv[i]] = i;
    __syncthreads();
    for (int k = tid; k < n; k += nt) pb[k] = rowat[k] >= 0 ? b[rowat[k]] : 0.0;
    __syncthreads();
    for (int k = 0; k < n; k++) {
        const double yk = __ddiv_rn(pb[k], Lx[Lp[k]]);
        if (tid == 0) y[k] = yk;
        for (int p = Lp[k] + 1 + tid; p < Lp[k + 1]; p += nt)
            pb[Li[p]] = __dsub_rn(pb[Li[p]], __dmul_rn(Lx[p], yk));
        __syncthreads();
    }
    // z overwrites pb (no longer needed).
    double* z = pb;
    for (int k = n - 1; k >= 0; k--) {
        const double zk = __ddiv_rn(y[k], Ux[Up[k + 1] - 1]);
        if (tid == 0) z[k] = zk;
        for (int p = Up[k] + tid; p < Up[k + 1] - 1; p += nt)
            y[Ui[p]] = __dsub_rn(y[Ui[p]], __dmul_rn(Ux[p], zk));
        __syncthreads();
    }
    for (int k = tid; k < n; k += nt) x[q ? q[k] : k] = z[k];
}

extern "C" int lusp_lu_factor_par_launch(int n, const int* Ap, const int* Ai, const double* Ax,
                                         const int* diagrow, int* Lp, int* Li, double* Lx,
                                         long Lcap, int* Up, int* Ui, double* Ux, long Ucap,
                                         int* pinv, int* xi, double* xg, int* lnnz, int* unnz,
                                         int* singular_out, void* stream) {
    const size_t bytes = LU_PAR_SHARED_BYTES(n);
    cudaError_t e = cudaFuncSetAttribute(lu_factor_par_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return (int)e;
    lu_factor_par_kernel<<<1, 256, bytes, (cudaStream_t)stream>>>(
        n, Ap, Ai, Ax, diagrow, Lp, Li, Lx, Lcap, Up, Ui, Ux, Ucap, pinv, xi, xg, lnnz, unnz,
        singular_out);
    return (int)cudaGetLastError();
}

extern "C" int lusp_trisolve_par_launch(int n, const int* Lp, const int* Li, const double* Lx,
                                        const int* Up, const int* Ui, const double* Ux,
                                        const int* pinv, const int* q, const double* b, double* x,
                                        int* work_i, double* work_d, void* stream) {
    trisolve_par_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(n, Lp, Li, Lx, Up, Ui, Ux, pinv, q, b,
                                                            x, work_i, work_d);
    return (int)cudaGetLastError();
}
