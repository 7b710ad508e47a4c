// kernels_batch.cu -- the batching form: thousands of independent dense
// systems of uneven order factored and solved by one persistent launch.
//
// Every system is lu2's augmented problem (row-major, b in the columns
// n..n+nrhs-1, lu2.c:28) and is solved with lu2's algorithm: partial pivoting
// with the first maximal |a| (lu2tlib.c:42-52), the pivot row scaled by
// 1/pivot (lu2tlib.c:1057-1059, lu2.c:551-552), right-looking updates that
// carry the right-hand sides along (lu2.c:1138), then the unit-upper back
// substitution (lu2.c:110-116).  x overwrites b.
//
// CTAs take systems from a queue ordered largest first (an atomic counter over
// a host-sorted order).  A system whose augmented matrix fits the shared
// memory budget is factored and solved there; larger ones run a blocked LU on
// the L2-resident matrix with the panel (all remaining rows x pw columns) in
// shared memory and the trailing update on the FP64 tensor cores (mma.sync
// m16n8k8) from the panel and a shared-memory copy of the U block.
#include <climits>

#include "lu2gpu_internal.cuh"

namespace lu2gpu {

constexpr int BATCH_LOAD_U = 4;  // global loads a thread keeps in flight when staging

// whole system in shared memory: S (n x nc, stride nc)
__device__ void batch_solve_smem(double *A, long ld, int n, int nrhs, double *S, int *info)
{
    const int nc = n + nrhs, T = blockDim.x, tid = threadIdx.x;
    // BATCH_LOAD_U loads in flight per thread
    for (int idx0 = tid; idx0 < n * nc; idx0 += BATCH_LOAD_U * T) {
        double v[BATCH_LOAD_U];
#pragma unroll
        for (int u = 0; u < BATCH_LOAD_U; u++) {
            const int idx = idx0 + u * T, r = idx / nc, c = idx - r * nc;
            v[u] = (idx < n * nc) ? A[(size_t)r * ld + c] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < BATCH_LOAD_U; u++)
            if (idx0 + u * T < n * nc) S[idx0 + u * T] = v[u];
    }
    __syncthreads();
    int first_zero = 0;
    for (int k = 0; k < n; k++) {
        // pivot search, row exchange and 1/pivot scaling by warp 0 alone
        // (warp-synchronous), then one barrier; the rank-1 update by all
        if (tid < 32) {
            const int lane = tid;
            double v = -1.0;
            int p = INT_MAX;
            for (int r = k + lane; r < n; r += 32) {
                const double a = fabs(S[r * nc + k]);
                if (a > v) {
                    v = a;
                    p = r;
                }
            }
            warp_argmax(v, p);
            if (p == INT_MAX) p = k;
            if (p != k)
                for (int c = lane; c < nc; c += 32) {
                    const double t = S[k * nc + c];
                    S[k * nc + c] = S[p * nc + c];
                    S[p * nc + c] = t;
                }
            __syncwarp();
            const double d = S[k * nc + k];
            if (d != 0.0) {
                const double inv = 1.0 / d;
                for (int c = k + 1 + lane; c < nc; c += 32) S[k * nc + c] *= inv;
            }
        }
        __syncthreads();
        const double d = S[k * nc + k];
        if (d == 0.0) {
            if (!first_zero) first_zero = k + 1;
            continue;
        }
        const int w = nc - k - 1, h = n - k - 1;
        for (int idx = tid; idx < h * w; idx += T) {
            const int r = k + 1 + idx / w, c = k + 1 + idx % w;
            S[r * nc + c] -= S[r * nc + k] * S[k * nc + c];
        }
        __syncthreads();
    }
    for (int j = n - 1; j >= 1; j--) {
        for (int idx = tid; idx < j * nrhs; idx += T) {
            const int i = idx / nrhs, q = idx - i * nrhs;
            S[i * nc + n + q] -= S[i * nc + j] * S[j * nc + n + q];
        }
        __syncthreads();
    }
    for (int idx = tid; idx < n * nrhs; idx += T) {
        const int r = idx / nrhs, q = idx - r * nrhs;
        A[(size_t)r * ld + n + q] = S[r * nc + n + q];
    }
    if (tid == 0) *info = first_zero;
}

__device__ __forceinline__ void batch_dmma(double (&c)[4], double a0, double a1, double a2, double a3, double b0,
                                           double b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

// blocked LU in global memory (L2-resident), panel of pw columns in shared memory
__device__ void batch_solve_blocked(double *A, long ld, int n, int nrhs, int pw, double *P, double *U, int *piv,
                                    double *dinv, BatchPlan &plan, int *info)
{
    __shared__ double s_pv[4];  // the panel warps' pivot candidates
    __shared__ int s_pi[4];
    const int nc = n + nrhs, T = blockDim.x, tid = threadIdx.x;
    // panel row stride pw + 1 (odd): the lanes of the panel factorization, one
    // row each, fall into different banks
    const int ps = pw + BATCH_PANEL_PAD;
    int first_zero = 0;
    for (int k0 = 0; k0 < n; k0 += pw) {
        const int w = min(pw, n - k0), rows = n - k0;
        // panel rows k0..n-1, columns k0..k0+w-1 -> P (rows x ps)
        for (int idx0 = tid; idx0 < rows * w; idx0 += BATCH_LOAD_U * T) {
            double v[BATCH_LOAD_U];
#pragma unroll
            for (int u = 0; u < BATCH_LOAD_U; u++) {
                const int idx = idx0 + u * T, r = idx / w, c = idx - r * w;
                v[u] = (idx < rows * w) ? A[(size_t)(k0 + r) * ld + k0 + c] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < BATCH_LOAD_U; u++) {
                const int idx = idx0 + u * T, r = idx / w, c = idx - r * w;
                if (idx < rows * w) P[r * ps + c] = v[u];
            }
        }
        __syncthreads();
        // the panel factored by the first NWP warps (up to 4): thread pt owns
        // the rows c + pt + k S (S = 32 NWP) of column c -- the same rows for
        // the pivot search of column c and the rank-1 step of column c - 1,
        // so it only reads rows it wrote itself; two named barriers of the S
        // threads per column (candidates in, pivot row swapped and scaled),
        // no CTA barrier; per element the same operations as a CTA-wide
        // elimination
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
                    const double a = fabs(P[r * ps + c]);
                    if (a > v) {
                        v = a;
                        p = r;
                    }
                }
                warp_argmax(v, p);
                if (lane == 0) {
                    s_pv[pw_] = v;
                    s_pi[pw_] = p;
                }
                asm volatile("bar.sync 1, %0;" ::"r"(S) : "memory");
                v = s_pv[0];
                p = s_pi[0];
                for (int q = 1; q < nwp; q++)
                    if (argmax_better(s_pv[q], s_pi[q], v, p)) {
                        v = s_pv[q];
                        p = s_pi[q];
                    }
                if (p == INT_MAX) p = c;
                if (tid < 32) {
                    if (lane == 0) piv[c] = p;
                    if (p != c)
                        for (int j = lane; j < w; j += 32) {
                            const double t = P[c * ps + j];
                            P[c * ps + j] = P[p * ps + j];
                            P[p * ps + j] = t;
                        }
                    __syncwarp();
                    const double d = P[c * ps + c];
                    const bool zero = (d == 0.0);
                    const double inv = zero ? 1.0 : 1.0 / d;
                    if (lane == 0) dinv[c] = inv;
                    __syncwarp();  // every lane has read the pivot before it is scaled
                    if (!zero)
                        for (int j = lane; j < w; j += 32)
                            if (j != c) P[c * ps + j] *= inv;
                    batch_plan_step(plan, c, p, w, lane);
                }
                asm volatile("bar.sync 1, %0;" ::"r"(S) : "memory");
                const bool zero = (P[c * ps + c] == 0.0);
                if (zero && !first_zero) first_zero = k0 + c + 1;
                if (!zero)
                    for (int r = c + 1 + tid; r < rows; r += S) {
                        const double l = P[r * ps + c];
                        for (int j = c + 1; j < w; j++) P[r * ps + j] -= l * P[c * ps + j];
                    }
            }
        }
        __syncthreads();  // (first_zero is tracked by the panel threads; thread 0 reports it)
        for (int idx = tid; idx < rows * w; idx += T) {
            const int r = idx / w, c = idx - r * w;
            A[(size_t)(k0 + r) * ld + k0 + c] = P[r * ps + c];
        }
        __syncthreads();
        // right part: the composed exchanges with 1/pivot scaling, then the
        // unit-lower solve of the U block rows, one thread per column
        // (lu2.c:524-581).  The gathers are issued 16 at a time, then the
        // displaced rows (loaded before U overwrites the rows they come from,
        // stored after every gather, since a gathered row may be one of them)
        const int cs = k0 + w, ne = plan.next;
        for (int j = cs + tid; j < nc; j += T) {
            double x[64];
            for (int q0 = 0; q0 < w; q0 += 16) {
                double v[16];
#pragma unroll
                for (int u = 0; u < 16; u++)
                    v[u] = q0 + u < w ? A[(size_t)(k0 + plan.blk[q0 + u]) * ld + j] : 0.0;
#pragma unroll
                for (int u = 0; u < 16; u++)
                    if (q0 + u < w) x[q0 + u] = v[u] * dinv[q0 + u];
            }
            for (int e0 = 0; e0 < ne; e0 += 16) {
                double v[16];
#pragma unroll
                for (int u = 0; u < 16; u++)
                    v[u] = e0 + u < ne ? A[(size_t)(k0 + plan.ext_src[e0 + u]) * ld + j] : 0.0;
#pragma unroll
                for (int u = 0; u < 16; u++)
                    if (e0 + u < ne) A[(size_t)(k0 + plan.ext_row[e0 + u]) * ld + j] = v[u];
            }
            for (int r = 1; r < w; r++) {
                double s = x[r];
                for (int l = 0; l < r; l++) s -= P[r * ps + l] * x[l];
                x[r] = s;
            }
            for (int c = 0; c < w; c++) A[(size_t)(k0 + c) * ld + j] = x[c];
        }
        __syncthreads();
        // trailing update A[k0+w.., cs..] -= L21 U12 on the FP64 tensor cores
        // (mma.sync m16n8k8 f64), in BATCH_U_CHUNK-column chunks of U12 staged in shared
        // memory; a warp takes 16 x 32 units (two per chunk row strip): C
        // fragments from global memory, -L21 fragments from the panel, U12
        // fragments from the chunk, K padded to a multiple of 8 with zeros
        const int h = n - cs;
        const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3, nwarps = T >> 5;
        const int ksteps = (w + 7) >> 3;
        const bool even = (cs & 1) == 0;  // 16-byte C accesses need an even column (always so: w = pw here)
        for (int c0 = cs; c0 < nc && h > 0; c0 += BATCH_U_CHUNK) {
            const int cw = min(BATCH_U_CHUNK, nc - c0);
            for (int idx = tid; idx < pw * BATCH_U_CHUNK; idx += T) {
                const int l = idx / BATCH_U_CHUNK, c = idx % BATCH_U_CHUNK;
                U[l * BATCH_U_STRIDE + c] = (l < w && c < cw) ? A[(size_t)(k0 + l) * ld + c0 + c] : 0.0;
            }
            __syncthreads();
            constexpr int UNB = BATCH_UNIT_COLS / 8;           // 8-column MMA blocks of a unit
            constexpr int PARTS = BATCH_U_CHUNK / BATCH_UNIT_COLS;  // units across a chunk's 16-row strip
            const int units = ((h + 15) >> 4) * PARTS;
            for (int u = warp; u < units; u += nwarps) {
                const int r0 = (u / PARTS) << 4, cb = (u % PARTS) * BATCH_UNIT_COLS;  // strip rows r0.., chunk columns cb..
                const int rl = r0 + g, rh = rl + 8;                // rows (of the trailing block) of c0,c1 / c2,c3
                double acc[UNB][4];
#pragma unroll
                for (int j = 0; j < UNB; j++) {
                    const int col = cb + 8 * j + 2 * t;  // chunk column of c0 / c2
#pragma unroll
                    for (int hh = 0; hh < 2; hh++) {
                        const int r = hh ? rh : rl;
                        double v0 = 0.0, v1 = 0.0;
                        if (r < h && col < cw) {
                            const double *cp = A + (size_t)(cs + r) * ld + c0 + col;
                            if (even && col + 1 < cw) {
                                const double2 v = *reinterpret_cast<const double2 *>(cp);
                                v0 = v.x;
                                v1 = v.y;
                            } else {
                                v0 = cp[0];
                                if (col + 1 < cw) v1 = cp[1];
                            }
                        }
                        acc[j][2 * hh] = v0;
                        acc[j][2 * hh + 1] = v1;
                    }
                }
                for (int kk = 0; kk < ksteps; kk++) {
                    const int ka = 8 * kk + t, kb = ka + 4;
                    const double *pl = P + (size_t)(w + rl) * ps, *ph = P + (size_t)(w + rh) * ps;
                    const double a0 = (rl < h && ka < w) ? -pl[ka] : 0.0;
                    const double a1 = (rh < h && ka < w) ? -ph[ka] : 0.0;
                    const double a2 = (rl < h && kb < w) ? -pl[kb] : 0.0;
                    const double a3 = (rh < h && kb < w) ? -ph[kb] : 0.0;
#pragma unroll
                    for (int j = 0; j < UNB; j++) {
                        const double b0 = U[ka * BATCH_U_STRIDE + cb + 8 * j + g];
                        const double b1 = U[kb * BATCH_U_STRIDE + cb + 8 * j + g];
                        batch_dmma(acc[j], a0, a1, a2, a3, b0, b1);
                    }
                }
#pragma unroll
                for (int j = 0; j < UNB; j++) {
                    const int col = cb + 8 * j + 2 * t;
#pragma unroll
                    for (int hh = 0; hh < 2; hh++) {
                        const int r = hh ? rh : rl;
                        if (r >= h || col >= cw) continue;
                        double *cp = A + (size_t)(cs + r) * ld + c0 + col;
                        if (even && col + 1 < cw) {
                            *reinterpret_cast<double2 *>(cp) = make_double2(acc[j][2 * hh], acc[j][2 * hh + 1]);
                        } else {
                            cp[0] = acc[j][2 * hh];
                            if (col + 1 < cw) cp[1] = acc[j][2 * hh + 1];
                        }
                    }
                }
            }
            __syncthreads();
        }
    }
    // back substitution with the unit upper factor (lu2.c:110-116), blocked by
    // 32 rows: y (n x nrhs) and each 32 x 32 diagonal block in shared memory
    // (reusing the panel's space); warp 0 solves the diagonal block
    // warp-synchronously (lane = row, the solved value passed by shuffle),
    // then the rows above are updated from their 32-wide row segments, four
    // threads per row on interleaved 16-byte column pairs
    double *Y = P;
    double *Ud = P + (size_t)n * nrhs;  // 32 x 33
    for (int idx = tid; idx < n * nrhs; idx += T) {
        const int r = idx / nrhs, q = idx - r * nrhs;
        Y[idx] = A[(size_t)r * ld + n + q];
    }
    const int warp = tid >> 5, lane = tid & 31, part = tid & 3;
    for (int jb = ((n - 1) / 32) * 32; jb >= 0; jb -= 32) {
        const int je = min(jb + 32, n), bw = je - jb;
        for (int idx = tid; idx < bw * bw; idx += T) {
            const int i = idx / bw, j = idx - i * bw;
            Ud[i * 33 + j] = A[(size_t)(jb + i) * ld + jb + j];
        }
        __syncthreads();
        if (warp == 0) {
            for (int q = 0; q < nrhs; q++) {
                double y = lane < bw ? Y[(jb + lane) * nrhs + q] : 0.0;
                for (int j = bw - 1; j >= 1; j--) {
                    const double yj = __shfl_sync(0xffffffffu, y, j);
                    if (lane < j) y -= Ud[lane * 33 + j] * yj;
                }
                if (lane < bw) Y[(jb + lane) * nrhs + q] = y;
            }
        }
        __syncthreads();
        // (jb, ld and the system's base are even / 16-byte aligned: jb > 0 rows
        // take one 16-byte load per column pair)
        for (int i0 = 0; i0 < jb; i0 += T >> 2) {
            const int i = i0 + (tid >> 2);
            double u[8];
#pragma unroll
            for (int e = 0; e < 8; e++) u[e] = 0.0;
            if (i < jb) {
                const double *row = A + (size_t)i * ld + jb + 2 * part;
#pragma unroll
                for (int jj = 0; jj < 4; jj++) {
                    const int c = 8 * jj + 2 * part;
                    if (c + 1 < bw) {
                        const double2 w = *reinterpret_cast<const double2 *>(row + 8 * jj);
                        u[2 * jj] = w.x;
                        u[2 * jj + 1] = w.y;
                    } else if (c < bw) {
                        u[2 * jj] = row[8 * jj];
                    }
                }
            }
            for (int q = 0; q < nrhs; q++) {
                double sacc = 0.0;
#pragma unroll
                for (int jj = 0; jj < 4; jj++) {
                    const int c = 8 * jj + 2 * part;
                    if (c < bw) sacc = fma(u[2 * jj], Y[(jb + c) * nrhs + q], sacc);
                    if (c + 1 < bw) sacc = fma(u[2 * jj + 1], Y[(jb + c + 1) * nrhs + q], sacc);
                }
                sacc += __shfl_xor_sync(0xffffffffu, sacc, 1);
                sacc += __shfl_xor_sync(0xffffffffu, sacc, 2);
                if (part == 0 && i < jb) Y[i * nrhs + q] -= sacc;
            }
        }
        __syncthreads();
    }
    for (int idx = tid; idx < n * nrhs; idx += T) {
        const int r = idx / nrhs, q = idx - r * nrhs;
        A[(size_t)r * ld + n + q] = Y[idx];
    }
    if (tid == 0) *info = first_zero;
}

__global__ void __launch_bounds__(512, 2) batch_lu_kernel(double *data, const BatchSys *sys, const int *order, int count, int *counter,
                                int *info, int pw, long smem_doubles)
{
    extern __shared__ double bsm[];
    __shared__ int s_next;
    __shared__ int s_piv[64];
    __shared__ double s_dinv[64];
    __shared__ BatchPlan s_plan;
    for (;;) {
        if (threadIdx.x == 0) s_next = atomicAdd(counter, 1);
        __syncthreads();
        const int q = s_next;
        __syncthreads();
        if (q >= count) break;
        const int i = order[q];
        const BatchSys S = sys[i];
        double *A = data + S.off;
        if ((long)S.n * (S.n + S.nrhs) <= smem_doubles) {
            batch_solve_smem(A, S.ld, S.n, S.nrhs, bsm, info + i);
        } else {
            // panel (n x pw) then the U chunk (pw x 64); the system's own panel
            // width when its size bucket has one
            const int pwi = S.pw ? S.pw : pw;
            batch_solve_blocked(A, S.ld, S.n, S.nrhs, pwi, bsm, bsm + (size_t)S.n * (pwi + BATCH_PANEL_PAD), s_piv,
                                s_dinv, s_plan, info + i);
        }
        __syncthreads();
    }
}

long batch_smem_doubles(const BatchSys *sys, int count, int pw)
{
    // blocked path of system i: its panel (n x (pw + pad)) then either the U
    // chunk (pw x BATCH_U_STRIDE) or, in the back substitution, y (n x nrhs)
    // then a 32 x 33 diagonal block; the in-shared-memory path uses whatever
    // this leaves
    long need = 0;
    for (int i = 0; i < count; i++) {
        const long pwi = sys[i].pw ? sys[i].pw : pw;
        const long tail = pwi * BATCH_U_STRIDE > 32 * 33 ? pwi * BATCH_U_STRIDE : 32 * 33;
        const long ps = pwi + BATCH_PANEL_PAD;
        const long w = sys[i].nrhs > ps ? sys[i].nrhs : ps;
        const long ni = (long)sys[i].n * w + tail;
        if (ni > need) need = ni;
    }
    return need;
}

cudaError_t batch_lu_grid(int threads, long smem_doubles, int ctas_per_sm, int count, int *grid)
{
    if (threads < 64 || threads > 512 || (threads & 31)) return cudaErrorInvalidValue;
    const size_t smem = (size_t)smem_doubles * sizeof(double);
    if (smem > BATCH_SMEM_MAX) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(batch_lu_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, BATCH_SMEM_MAX);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    int occ = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_lu_kernel, threads, smem)) != cudaSuccess)
        return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    if (ctas_per_sm > occ || ctas_per_sm < 1) ctas_per_sm = occ;
    int g = sms * ctas_per_sm;
    *grid = g > count ? count : g;
    return cudaSuccess;
}

cudaError_t launch_batch_lu(double *data, const BatchSys *sys, const int *order, int count, int *counter, int *info,
                            long smem_doubles, int pw, int threads, int grid, cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    if (pw < 16 || pw > 64 || threads < 64 || threads > 512 || (threads & 31) || grid < 1 ||
        (size_t)smem_doubles * sizeof(double) > BATCH_SMEM_MAX)
        return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    count_launch();
    batch_lu_kernel<<<grid, threads, (size_t)smem_doubles * sizeof(double), st>>>(data, sys, order, count, counter,
                                                                                   info, pw, smem_doubles);
    return cudaGetLastError();
}

// HPL scaled residual of every solved system against its original copy:
// out[i] = max over right-hand sides of ||A x - b||_inf / (eps (||A||_inf ||x||_inf + ||b||_inf) n)
__global__ void batch_residual_kernel(const double *orig, const double *solved, const BatchSys *sys, int count,
                                      double *out)
{
    __shared__ double s_r[32], s_a[32], s_x[32], s_b[32];
    for (int i = blockIdx.x; i < count; i += gridDim.x) {
        const BatchSys S = sys[i];
        const double *A = orig + S.off, *X = solved + S.off;
        double worst = 0.0;
        for (int q = 0; q < S.nrhs; q++) {
            double rmax = 0, amax = 0, xmax = 0, bmax = 0;
            for (int r = threadIdx.x; r < S.n; r += blockDim.x) {
                double s = 0, sa = 0;
                for (int c = 0; c < S.n; c++) {
                    const double a = A[(size_t)r * S.ld + c];
                    s = fma(a, X[(size_t)c * S.ld + S.n + q], s);
                    sa += fabs(a);
                }
                const double b = A[(size_t)r * S.ld + S.n + q];
                rmax = fmax(rmax, fabs(s - b));
                amax = fmax(amax, sa);
                bmax = fmax(bmax, fabs(b));
                xmax = fmax(xmax, fabs(X[(size_t)r * S.ld + S.n + q]));
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
                amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
                xmax = fmax(xmax, __shfl_xor_sync(0xffffffffu, xmax, o));
                bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
            }
            const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
            if (lane == 0) {
                s_r[warp] = rmax;
                s_a[warp] = amax;
                s_x[warp] = xmax;
                s_b[warp] = bmax;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                for (int w2 = 1; w2 < nw; w2++) {
                    rmax = fmax(rmax, s_r[w2]);
                    amax = fmax(amax, s_a[w2]);
                    xmax = fmax(xmax, s_x[w2]);
                    bmax = fmax(bmax, s_b[w2]);
                }
                const double h = rmax / (1.1102230246251565e-16 * (amax * xmax + bmax) * S.n);
                worst = fmax(worst, h);
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) out[i] = worst;
    }
}

cudaError_t launch_batch_residual(const double *orig, const double *solved, const BatchSys *sys, int count,
                                  double *out, cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    count_launch();
    batch_residual_kernel<<<count < 148 * 8 ? count : 148 * 8, 256, 0, st>>>(orig, solved, sys, count, out);
    return cudaGetLastError();
}

// system i of a batch: lu2's stream (randomsetmat) with seed seeds[i], or
// seed_base + i without a seed list
__global__ void batch_generate_kernel(double *data, const BatchSys *sys, int count, unsigned long long seed_base,
                                      const long long *seeds)
{
    for (int i = blockIdx.x; i < count; i += gridDim.x) {
        const BatchSys S = sys[i];
        double *A = data + S.off;
        const unsigned long long seed = seeds ? (unsigned long long)seeds[i] : seed_base + i;
        const unsigned long long xs = ((seed & 0xffffffffull) << 16) | 0x330Eull;
        const long total = (long)S.n * (S.n + 1) + (long)S.n * (S.nrhs - 1);
        for (long q = threadIdx.x; q < total; q += blockDim.x) {
            unsigned long long k = q + 1, aa = 1, cc = 0, ba = 0x5DEECE66Dull, bc = 0xBull;
            const unsigned long long M = (1ull << 48) - 1;
            while (k) {
                if (k & 1) {
                    cc = (ba * cc + bc) & M;
                    aa = (ba * aa) & M;
                }
                bc = (ba * bc + bc) & M;
                ba = (ba * ba) & M;
                k >>= 1;
            }
            const double v = (double)((aa * xs + cc) & M) * (1.0 / 281474976710656.0) - 0.5;
            long r, c;
            if (q < (long)S.n * (S.n + 1)) {
                r = q / (S.n + 1);
                c = q - r * (S.n + 1);
            } else {
                const long e = q - (long)S.n * (S.n + 1);
                c = S.n + 1 + e / S.n;
                r = e % S.n;
            }
            A[(size_t)r * S.ld + c] = v;
        }
    }
}

cudaError_t launch_batch_generate(double *data, const BatchSys *sys, int count, unsigned long long seed_base,
                                  const long long *seeds, cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    count_launch();
    batch_generate_kernel<<<count < 148 * 16 ? count : 148 * 16, 256, 0, st>>>(data, sys, count, seed_base, seeds);
    return cudaGetLastError();
}

}  // namespace lu2gpu
