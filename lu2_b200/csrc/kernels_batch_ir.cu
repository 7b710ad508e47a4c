// kernels_batch_ir.cu -- the batching form's FP32-LU + FP64 iterative
// refinement variant: every system's FP64 augmented matrix (left unchanged
// until x is written into its b columns) is converted to FP32, factored in
// FP32, and refined in FP64 -- r = b - A x from the FP64 matrix, the
// correction solved with the FP32 factors -- until every right-hand side has
// an HPL scaled residual below 16 (or max_iter corrections).
//
// Factor storage follows lu2's elimination (lu2.c:541-554, lu2tlib.c:1057-
// 1059): the pivot row is scaled by 1/pivot right of the diagonal (a unit
// upper U'), the columns below keep the unscaled multipliers times the pivot
// (L' lower with the pivots on its diagonal).  Unlike lu2, whose solve rides
// along as augmented columns, the refinement needs the factors for new
// right-hand sides, so rows are exchanged over their full width (LAPACK
// order): P A = L' U', solved as y = L'^{-1} P r, d = U'^{-1} y.
//
// One CTA per system from a largest-first queue, as in the FP64 variant.
// Systems whose FP32 matrix fits shared memory are factored and solved
// there; larger ones are factored blocked in their FP32 slot of the work
// arena (panel of pw columns in shared memory) and solved from it.
#include <climits>

#include "lu2gpu_internal.cuh"

namespace lu2gpu {

// FP32 factorization of F (n x n, stride fs) held in shared memory: per
// column warp 0 alone (warp-synchronously) searches the pivot, exchanges the
// full rows and scales the pivot row, then after one barrier every thread
// takes part in the rank-1 update -- two barriers per column
__device__ void ir_factor_smem(float *F, int n, int fs, int *piv, int *first_zero)
{
    const int T = blockDim.x, tid = threadIdx.x;
    for (int k = 0; k < n; k++) {
        if (tid < 32) {
            const int lane = tid;
            double v = -1.0;
            int p = INT_MAX;
            for (int r = k + lane; r < n; r += 32) {
                const double a = fabsf(F[r * fs + k]);
                if (a > v) {
                    v = a;
                    p = r;
                }
            }
            warp_argmax(v, p);
            if (p == INT_MAX) p = k;
            if (lane == 0) piv[k] = p;
            if (p != k)
                for (int c = lane; c < n; c += 32) {
                    const float t = F[k * fs + c];
                    F[k * fs + c] = F[p * fs + c];
                    F[p * fs + c] = t;
                }
            __syncwarp();
            const float d = F[k * fs + k];
            __syncwarp();  // every lane has read the pivot before the row is scaled
            if (d != 0.f) {
                const float inv = 1.f / d;
                for (int c = k + 1 + lane; c < n; c += 32) F[k * fs + c] *= inv;
            } else if (lane == 0 && !*first_zero) {
                *first_zero = k + 1;
            }
        }
        __syncthreads();
        if (F[k * fs + k] == 0.f) continue;  // (uniform: every thread reads the same pivot)
        const int w = n - k - 1;
        for (int idx = tid; idx < w * w; idx += T) {
            const int r = k + 1 + idx / w, c = k + 1 + idx % w;
            F[r * fs + c] -= F[r * fs + k] * F[k * fs + c];
        }
        __syncthreads();
    }
}

// FP32 factorization of F (n x n, stride n) in global memory, panel of pw
// columns staged in shared memory (P: rows x (pw+1), U: pw x 64).  The panel
// is factored by the first NWP warps (up to 4), thread pt owning the panel
// rows c + pt + k S (S = 32 NWP) for both the pivot search of column c and
// the rank-1 step of column c - 1, with two named barriers of the S threads
// per column; warp 0 composes the panel's row exchanges into one plan, which
// the columns left of the panel (full-width exchanges) and the right part
// then apply with independent loads instead of one dependent swap per pivot.
__device__ void ir_factor_blocked(float *F, int n, int pw, float *P, float *U, int *piv, float *dinv,
                                  int *first_zero, double *s_v, int *s_i, BatchPlan &plan)
{
    const int T = blockDim.x, tid = threadIdx.x;
    const int ps = pw + 1;  // odd panel row stride: a column's rows fall in distinct banks
    for (int k0 = 0; k0 < n; k0 += pw) {
        const int w = min(pw, n - k0), rows = n - k0;
        for (int idx = tid; idx < rows * w; idx += T) {
            const int r = idx / w, c = idx - r * w;
            P[r * ps + c] = F[(size_t)(k0 + r) * n + k0 + c];
        }
        __syncthreads();
        const int nwp = min(4, T >> 5), S = 32 * nwp;
        if (tid < S) {
            const int lane = tid & 31, pw_ = tid >> 5;
            if (tid < 32) {
                for (int q = lane; q < w; q += 32) plan.blk[q] = q;
                if (lane == 0) plan.next = 0;
                __syncwarp();
            }
            for (int c = 0; c < w; c++) {
                double v = -1.0;
                int p = INT_MAX;
                for (int r = c + tid; r < rows; r += S) {
                    const double a = fabsf(P[r * ps + c]);
                    if (a > v) {
                        v = a;
                        p = r;
                    }
                }
                warp_argmax(v, p);
                if (lane == 0) {
                    s_v[pw_] = v;
                    s_i[pw_] = p;
                }
                asm volatile("bar.sync 1, %0;" ::"r"(S) : "memory");
                v = s_v[0];
                p = s_i[0];
                for (int q = 1; q < nwp; q++)
                    if (argmax_better(s_v[q], s_i[q], v, p)) {
                        v = s_v[q];
                        p = s_i[q];
                    }
                if (p == INT_MAX) p = c;
                if (tid < 32) {
                    if (lane == 0) piv[k0 + c] = k0 + p;
                    if (p != c)
                        for (int j = lane; j < w; j += 32) {
                            const float t = P[c * ps + j];
                            P[c * ps + j] = P[p * ps + j];
                            P[p * ps + j] = t;
                        }
                    __syncwarp();
                    const float d = P[c * ps + c];
                    const bool zero = (d == 0.f);
                    const float inv = zero ? 1.f : 1.f / d;
                    if (lane == 0) dinv[c] = inv;
                    __syncwarp();  // every lane has read the pivot before the row is scaled
                    if (!zero)
                        for (int j = c + 1 + lane; j < w; j += 32) P[c * ps + j] *= inv;
                    batch_plan_step(plan, c, p, w, lane);
                }
                asm volatile("bar.sync 1, %0;" ::"r"(S) : "memory");
                const bool zero = (P[c * ps + c] == 0.f);
                if (zero && tid == 0 && !*first_zero) *first_zero = k0 + c + 1;
                if (!zero)
                    for (int r = c + 1 + tid; r < rows; r += S) {
                        const float l = P[r * ps + c];
                        for (int j = c + 1; j < w; j++) P[r * ps + j] -= l * P[c * ps + j];
                    }
            }
        }
        __syncthreads();
        for (int idx = tid; idx < rows * w; idx += T) {
            const int r = idx / w, c = idx - r * w;
            F[(size_t)(k0 + r) * n + k0 + c] = P[r * ps + c];
        }
        // the composed exchanges on the columns left of the panel (full-width
        // rows) and, with the unit-lower solve and the 1/pivot scaling, on the
        // right part, one thread per column: every gather first (16 loads in
        // flight), then the displaced rows (read before the rows they come
        // from are rewritten, written after every gather, since a gathered row
        // may be one of them), then the panel's rows
        const int cs = k0 + w, ne = plan.next, nleft = k0, ncols = k0 + (n - cs);
        for (int jj = tid; jj < ncols; jj += T) {
            const int j = jj < nleft ? jj : cs + (jj - nleft);
            float x[64];
            for (int q0 = 0; q0 < w; q0 += 16) {
                float v[16];
#pragma unroll
                for (int u = 0; u < 16; u++) v[u] = q0 + u < w ? F[(size_t)(k0 + plan.blk[q0 + u]) * n + j] : 0.f;
#pragma unroll
                for (int u = 0; u < 16; u++)
                    if (q0 + u < w) x[q0 + u] = v[u];
            }
            for (int e0 = 0; e0 < ne; e0 += 16) {
                float v[16];
#pragma unroll
                for (int u = 0; u < 16; u++)
                    v[u] = e0 + u < ne ? F[(size_t)(k0 + plan.ext_src[e0 + u]) * n + j] : 0.f;
#pragma unroll
                for (int u = 0; u < 16; u++)
                    if (e0 + u < ne) F[(size_t)(k0 + plan.ext_row[e0 + u]) * n + j] = v[u];
            }
            if (jj >= nleft)
                for (int r = 0; r < w; r++) {
                    float s = x[r];
                    for (int l = 0; l < r; l++) s -= P[r * ps + l] * x[l];
                    x[r] = s * dinv[r];
                }
            for (int c = 0; c < w; c++) F[(size_t)(k0 + c) * n + j] = x[c];
        }
        __syncthreads();
        // trailing update F[cs.., cs..] -= L21 U12 in 64-column chunks
        const int h = n - cs;
        for (int c0 = cs; c0 < n && h > 0; c0 += 64) {
            const int cw = min(64, n - c0);
            for (int idx = tid; idx < w * 64; idx += T) {
                const int l = idx >> 6, c = idx & 63;
                U[l * 64 + c] = (c < cw) ? F[(size_t)(k0 + l) * n + c0 + c] : 0.f;
            }
            __syncthreads();
            const int tx = tid & 15, ty = tid >> 4, tys = T >> 4;
            for (int rb = ty * 4; rb < h; rb += tys * 4) {
                float acc[4][4] = {};
                for (int l = 0; l < w; l++) {
                    float av[4], bv[4];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        av[i] = (rb + i < h) ? P[(w + rb + i) * ps + l] : 0.f;
                        bv[i] = U[l * 64 + tx * 4 + i];
                    }
#pragma unroll
                    for (int i = 0; i < 4; i++)
#pragma unroll
                        for (int q = 0; q < 4; q++) acc[i][q] = fmaf(av[i], bv[q], acc[i][q]);
                }
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    if (rb + i >= h) break;
                    float *row = F + (size_t)(cs + rb + i) * n + c0;
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        if (tx * 4 + q < cw) row[tx * 4 + q] -= acc[i][q];
                }
            }
            __syncthreads();
        }
    }
}

// V (n x r, row-major, shared memory) = U'^{-1} L'^{-1} P V with the FP32 factors F
// (stride n, shared or global memory); blocks of 32 rows: one warp solves the
// diagonal block, every thread updates the rows beyond it
__device__ void ir_solve(const float *F, int n, int fs, const int *piv, float *V, int r)
{
    const int T = blockDim.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int q = tid; q < r; q += T)
        for (int k = 0; k < n; k++) {
            const int p = piv[k];
            if (p != k) {
                const float t = V[k * r + q];
                V[k * r + q] = V[p * r + q];
                V[p * r + q] = t;
            }
        }
    __syncthreads();
    // forward: y_k = (v_k - sum_{j<k} L'_kj y_j) / L'_kk
    for (int b0 = 0; b0 < n; b0 += 32) {
        const int bw = min(32, n - b0);
        if (warp == 0)
            for (int q = 0; q < r; q++) {
                float v = lane < bw ? V[(b0 + lane) * r + q] : 0.f;
                for (int k = 0; k < bw; k++) {
                    float yk = __shfl_sync(0xffffffffu, v, k);
                    yk /= F[(size_t)(b0 + k) * fs + b0 + k];
                    if (lane == k) v = yk;
                    if (lane > k && lane < bw) v -= F[(size_t)(b0 + lane) * fs + b0 + k] * yk;
                }
                if (lane < bw) V[(b0 + lane) * r + q] = v;
            }
        __syncthreads();
        for (int idx = tid; idx < (n - b0 - bw) * r; idx += T) {
            const int i = b0 + bw + idx / r, q = idx % r;
            const float *row = F + (size_t)i * fs + b0;
            float s = 0.f;
            for (int k = 0; k < bw; k++) s = fmaf(row[k], V[(b0 + k) * r + q], s);
            V[i * r + q] -= s;
        }
        __syncthreads();
    }
    // backward: x_k = y_k - sum_{j>k} U'_kj x_j
    for (int be = n; be > 0; be -= 32) {
        const int b0 = max(0, be - 32), bw = be - b0;
        if (warp == 0)
            for (int q = 0; q < r; q++) {
                float v = lane < bw ? V[(b0 + lane) * r + q] : 0.f;
                for (int k = bw - 1; k >= 0; k--) {
                    const float xk = __shfl_sync(0xffffffffu, v, k);
                    if (lane < k) v -= F[(size_t)(b0 + lane) * fs + b0 + k] * xk;
                }
                if (lane < bw) V[(b0 + lane) * r + q] = v;
            }
        __syncthreads();
        for (int idx = tid; idx < b0 * r; idx += T) {
            const int i = idx / r, q = idx % r;
            const float *row = F + (size_t)i * fs + b0;
            float s = 0.f;
            for (int k = 0; k < bw; k++) s = fmaf(row[k], V[(b0 + k) * r + q], s);
            V[i * r + q] -= s;
        }
        __syncthreads();
    }
}

// R = B - A X (FP64, warp per row) and the HPL norms: per right-hand side
// max|r|, max|x|; with `first`, also max|b| and ||A||_inf
__device__ void ir_residual(const double *A, long ld, int n, int r, const double *X, double *R, bool first,
                            double *s_red, double *rmax, double *xmax, double *bmax, double *anorm)
{
    const int T = blockDim.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = T >> 5;
    double my_r[IR_MAX_RHS], my_b[IR_MAX_RHS], my_a = 0.0;
    for (int q = 0; q < IR_MAX_RHS; q++) my_r[q] = my_b[q] = 0.0;
    for (int i = warp; i < n; i += nw) {
        const double *row = A + (size_t)i * ld;
        double s[IR_MAX_RHS], sa = 0.0;
        for (int q = 0; q < IR_MAX_RHS; q++) s[q] = 0.0;
        for (int j = lane; j < n; j += 32) {
            const double a = row[j];
            sa += fabs(a);
            for (int q = 0; q < r; q++) s[q] = fma(a, X[(size_t)j * r + q], s[q]);
        }
        for (int o = 16; o > 0; o >>= 1) {
            sa += __shfl_xor_sync(0xffffffffu, sa, o);
            for (int q = 0; q < r; q++) s[q] += __shfl_xor_sync(0xffffffffu, s[q], o);
        }
        if (lane == 0) {
            my_a = fmax(my_a, sa);
            for (int q = 0; q < r; q++) {
                const double b = row[n + q];
                const double res = b - s[q];
                R[(size_t)i * r + q] = res;
                my_r[q] = fmax(my_r[q], fabs(res));
                my_b[q] = fmax(my_b[q], fabs(b));
            }
        }
    }
    // block maxima (lane 0 of every warp holds partials); s_red: 32 x (2 r + 1)
    const int stride = 2 * IR_MAX_RHS + 1;
    if (lane == 0) {
        for (int q = 0; q < r; q++) {
            s_red[warp * stride + q] = my_r[q];
            s_red[warp * stride + IR_MAX_RHS + q] = my_b[q];
        }
        s_red[warp * stride + 2 * IR_MAX_RHS] = my_a;
    }
    __syncthreads();
    if (tid < r) {
        double m1 = 0.0, m2 = 0.0, m3 = 0.0;
        for (int w = 0; w < nw; w++) {
            m1 = fmax(m1, s_red[w * stride + tid]);
            m2 = fmax(m2, s_red[w * stride + IR_MAX_RHS + tid]);
            m3 = fmax(m3, s_red[w * stride + 2 * IR_MAX_RHS]);
        }
        rmax[tid] = m1;
        if (first) {
            bmax[tid] = m2;
            if (tid == 0) *anorm = m3;
        }
        double xm = 0.0;
        for (int i = 0; i < n; i++) xm = fmax(xm, fabs(X[(size_t)i * r + tid]));
        xmax[tid] = xm;
    }
    __syncthreads();
}

__global__ void batch_ir_kernel(double *data, const BatchSys *sys, const long long *woff, uint8_t *arena,
                                const int *order, int count, int *counter, int *info, int *iters, int pw,
                                long smem_floats, int max_iter)
{
    extern __shared__ float ism[];
    __shared__ double s_v[32];
    __shared__ int s_i[32];
    __shared__ int s_next, s_zero, s_done;
    __shared__ float s_dinv[64];
    __shared__ BatchPlan s_plan;
    __shared__ double s_red[32 * (2 * IR_MAX_RHS + 1)];
    __shared__ double s_rmax[IR_MAX_RHS], s_xmax[IR_MAX_RHS], s_bmax[IR_MAX_RHS], s_anorm;
    const int T = blockDim.x, tid = threadIdx.x;
    for (;;) {
        if (tid == 0) s_next = atomicAdd(counter, 1);
        __syncthreads();
        const int qi = s_next;
        __syncthreads();
        if (qi >= count) break;
        const int si = order[qi];
        const BatchSys S = sys[si];
        const int n = S.n, r = S.nrhs;
        double *A = data + S.off;
        uint8_t *w = arena + woff[si];
        float *Fg = reinterpret_cast<float *>(w);
        int *piv = reinterpret_cast<int *>(w + ir_align16((size_t)n * n * 4));
        double *X = reinterpret_cast<double *>(w + ir_align16((size_t)n * n * 4) + ir_align16((size_t)n * 4));
        double *R = X + (size_t)n * r;
        // in shared memory with an odd row stride (a column's rows in distinct banks)
        const int fso = n | 1;
        const bool in_smem = (long)n * fso + (long)n * r <= smem_floats;
        const int fs = in_smem ? fso : n;
        float *F = in_smem ? ism : Fg;
        float *V = in_smem ? ism + (size_t)n * fs : ism + (size_t)n * (pw + 1) + (size_t)pw * 64;
        if (tid == 0) s_zero = 0;
        for (int idx = tid; idx < n * n; idx += T) {
            const int i = idx / n, j = idx - i * n;
            F[(size_t)i * fs + j] = (float)A[(size_t)i * S.ld + j];
        }
        __syncthreads();
        if (in_smem)
            ir_factor_smem(F, n, fs, piv, &s_zero);
        else
            ir_factor_blocked(F, n, pw, ism, ism + (size_t)n * (pw + 1), piv, s_dinv, &s_zero, s_v, s_i, s_plan);
        __syncthreads();
        int it = 0;
        if (s_zero == 0) {
            // x_0 = 0, r_0 = b
            for (int idx = tid; idx < n * r; idx += T) {
                const int i = idx / r, q = idx - i * r;
                X[idx] = 0.0;
                R[idx] = A[(size_t)i * S.ld + n + q];
            }
            __syncthreads();
            ir_residual(A, S.ld, n, r, X, R, true, s_red, s_rmax, s_xmax, s_bmax, &s_anorm);
            for (it = 1; it <= max_iter; it++) {
                for (int idx = tid; idx < n * r; idx += T) V[idx] = (float)R[idx];
                __syncthreads();
                ir_solve(F, n, fs, piv, V, r);
                for (int idx = tid; idx < n * r; idx += T) X[idx] += (double)V[idx];
                __syncthreads();
                ir_residual(A, S.ld, n, r, X, R, false, s_red, s_rmax, s_xmax, s_bmax, &s_anorm);
                if (tid == 0) {
                    bool ok = true;
                    for (int q = 0; q < r; q++) {
                        const double h = s_rmax[q] / (1.1102230246251565e-16 * (s_anorm * s_xmax[q] + s_bmax[q]) * n);
                        if (!(h < 16.0)) ok = false;
                    }
                    s_done = ok;
                }
                __syncthreads();
                if (s_done) break;
            }
            if (it > max_iter) it = max_iter;
            for (int idx = tid; idx < n * r; idx += T) {
                const int i = idx / r, q = idx - i * r;
                A[(size_t)i * S.ld + n + q] = X[idx];
            }
        }
        if (tid == 0) {
            info[si] = s_zero;
            iters[si] = it;
        }
        __syncthreads();
    }
}

long batch_ir_smem_floats(const BatchSys *sys, int count, int pw, long floor_floats)
{
    long need = floor_floats;
    for (int i = 0; i < count; i++) {
        const long b = (long)sys[i].n * (pw + 1) + (long)pw * 64 + (long)sys[i].n * sys[i].nrhs;
        if (b > need) need = b;
    }
    return need;
}

cudaError_t batch_ir_grid(int threads, long smem_floats, int ctas_per_sm, int count, int *grid)
{
    if (threads < 64 || threads > 1024 || (threads & 31)) return cudaErrorInvalidValue;
    const size_t smem = (size_t)smem_floats * sizeof(float);
    if (smem > BATCH_SMEM_MAX) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(batch_ir_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, BATCH_SMEM_MAX);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    int occ = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_ir_kernel, threads, smem)) != cudaSuccess)
        return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    if (ctas_per_sm > occ || ctas_per_sm < 1) ctas_per_sm = occ;
    const int g = sms * ctas_per_sm;
    *grid = g > count ? count : g;
    return cudaSuccess;
}

cudaError_t launch_batch_ir(double *data, const BatchSys *sys, const long long *woff, uint8_t *arena,
                            const int *order, int count, int *counter, int *info, int *iters, long smem_floats, int pw,
                            int threads, int grid, int max_iter, cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    if (pw < 16 || pw > 64 || threads < 64 || threads > 1024 || (threads & 31) || grid < 1 || max_iter < 1 ||
        (size_t)smem_floats * sizeof(float) > BATCH_SMEM_MAX)
        return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    count_launch();
    batch_ir_kernel<<<grid, threads, (size_t)smem_floats * sizeof(float), st>>>(
        data, sys, woff, arena, order, count, counter, info, iters, pw, smem_floats, max_iter);
    return cudaGetLastError();
}

}  // namespace lu2gpu
