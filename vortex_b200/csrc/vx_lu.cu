// vx_lu.cu — the panel system's inverse by a blocked LU factorisation with
// partial pivoting (gj_pivot 3), for bodies that do not need the reference's
// Gauss-Jordan pivot rule reproduced: about (2/3 + 2) n^3 FP64 operations in
// four kernels per block of 32 columns instead of 2n launches that each
// sweep the whole augmented matrix.
//
// Factorisation P A = L U (L unit lower, U upper), right-looking, panels of
// LU_B columns:
//   k_lu_panel   one block factorises the panel (n - k0 rows, LU_B columns):
//                per column the pivot (largest |a|, lowest row on a tie),
//                the swap inside the panel, the multipliers and the update
//                of the panel's later columns;
//   k_lu_swap    the panel's row swaps applied to every column outside it;
//   k_lu_trsm_l  U12 = L11^-1 A12 (one thread per column of A12);
//   k_gemm_sub   A22 -= L21 U12.
// Inverse: X = A^-1 solves L U X = P, by the same block steps over the n
// right-hand sides: forward (Y = L^-1 P) and backward (X = U^-1 Y).
// A pivot below 1e-12 sets *flag (the system is reported singular), as in
// the reference's inversion.
#include "vx_internal.cuh"

constexpr int LU_B = 32;       // panel width
constexpr int LU_T = 1024;     // threads of the panel block
constexpr int GM = 64;         // output tile of k_gemm_sub: GM x GM, k depth LU_B
constexpr int GT = 256;

__device__ __forceinline__ void lu_argmax(const double *A, long long n, long long col, long long r0, double *sv,
                                          int *si, double &best, long long &row) {
    double mv = -1.0;
    long long mi = n;
    for (long long i = r0 + threadIdx.x; i < n; i += blockDim.x) {
        const double a = fabs(A[i * n + col]);
        if (a > mv) { mv = a; mi = i; }
    }
    sv[threadIdx.x] = mv;
    si[threadIdx.x] = (int)mi;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            const double a = sv[threadIdx.x + o];
            const int ai = si[threadIdx.x + o];
            if (a > sv[threadIdx.x] || (a == sv[threadIdx.x] && ai < si[threadIdx.x])) {
                sv[threadIdx.x] = a;
                si[threadIdx.x] = ai;
            }
        }
        __syncthreads();
    }
    best = sv[0];
    row = si[0];
    __syncthreads();
}

// Panel k0 .. k0 + kb - 1 of the n x n row-major A (rows k0 .. n-1).
VX_DEVK void k_lu_panel_body(VxBlkB<LU_T, 0> vb, double *A, long long n, long long k0, int kb, int *piv, int *flag) {
    __shared__ double sv[LU_T];
    __shared__ int si[LU_T];
    if (*flag) return;
    for (int c = 0; c < kb; ++c) {
        const long long col = k0 + c;
        double best;
        long long p;
        lu_argmax(A, n, col, col, sv, si, best, p);
        if (!(best >= 1e-12)) {
            if (threadIdx.x == 0) *flag = 1;
            return;
        }
        if (threadIdx.x == 0) piv[col] = (int)p;
        if (p != col)
            for (int j = threadIdx.x; j < kb; j += blockDim.x) {
                const double t = A[col * n + k0 + j];
                A[col * n + k0 + j] = A[p * n + k0 + j];
                A[p * n + k0 + j] = t;
            }
        __syncthreads();
        const double d = A[col * n + col];
        for (long long i = col + 1 + threadIdx.x; i < n; i += blockDim.x) A[i * n + col] /= d;
        __syncthreads();
        const int w = kb - c - 1;   // later columns of the panel
        if (w > 0)
            for (long long e = threadIdx.x; e < (n - col - 1) * w; e += blockDim.x) {
                const long long i = col + 1 + e / w, j = col + 1 + e % w;
                A[i * n + j] -= A[i * n + col] * A[col * n + j];
            }
        __syncthreads();
    }
}
__global__ void __launch_bounds__(LU_T) k_lu_panel(double *A, long long n, long long k0, int kb, int *piv, int *flag) {
    VX_PDL_WAIT();
    k_lu_panel_body(VxBlkB<LU_T, 0>{blockIdx.x, gridDim.x}, A, n, k0, kb, piv, flag);
}

// The swaps of rows k0 .. k0 + kb - 1 (in order) on the columns outside the
// panel of A (n x n), and on every column of B (n x nb, may be null).
VX_DEVK void k_lu_swap_body(VxBlk vb, double *A, long long n, long long k0, int kb, const int *piv, const int *flag) {
    if (*flag) return;
    for (long long j = vb.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)vb.n * blockDim.x) {
        if (j >= k0 && j < k0 + kb) continue;
        for (int c = 0; c < kb; ++c) {
            const long long r = k0 + c, p = piv[r];
            if (p != r) {
                const double t = A[r * n + j];
                A[r * n + j] = A[p * n + j];
                A[p * n + j] = t;
            }
        }
    }
}
__global__ void k_lu_swap(double *A, long long n, long long k0, int kb, const int *piv, const int *flag) {
    VX_PDL_WAIT();
    k_lu_swap_body(VxBlk{blockIdx.x, gridDim.x}, A, n, k0, kb, piv, flag);
}

// Triangular solve on the block rows r0 .. r0 + kb - 1 of X (n x n), for
// the columns j in [j0, n): lower (unit diagonal, forward) or upper
// (backward, dividing by the diagonal) with the kb x kb diagonal block of T
// (n x n) at (r0, r0), staged in shared memory.
template <bool LOWER>
VX_DEVK void k_lu_trsm_body(VxBlkB<256, 0> vb, const double *T, double *X, long long n, long long r0, int kb,
                            long long j0, const int *flag) {
    __shared__ double t[LU_B][LU_B + 1];
    if (*flag) return;
    for (int e = threadIdx.x; e < kb * kb; e += blockDim.x) t[e / kb][e % kb] = T[(r0 + e / kb) * n + r0 + e % kb];
    __syncthreads();
    for (long long j = j0 + vb.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)vb.n * blockDim.x) {
        double x[LU_B];
#pragma unroll
        for (int r = 0; r < LU_B; ++r) x[r] = r < kb ? X[(r0 + r) * n + j] : 0.0;
        if (LOWER) {
#pragma unroll
            for (int r = 0; r < LU_B; ++r)
#pragma unroll
                for (int q = 0; q < r; ++q) x[r] -= t[r][q] * x[q];
        } else {
#pragma unroll
            for (int r = LU_B - 1; r >= 0; --r) {
                if (r >= kb) continue;
#pragma unroll
                for (int q = r + 1; q < LU_B; ++q)
                    if (q < kb) x[r] -= t[r][q] * x[q];
                x[r] /= t[r][r];
            }
        }
#pragma unroll
        for (int r = 0; r < LU_B; ++r)
            if (r < kb) X[(r0 + r) * n + j] = x[r];
    }
}
template <bool LOWER>
__global__ void __launch_bounds__(256) k_lu_trsm(const double *T, double *X, long long n, long long r0, int kb,
                                                 long long j0, const int *flag) {
    VX_PDL_WAIT();
    k_lu_trsm_body<LOWER>(VxBlkB<256, 0>{blockIdx.x, gridDim.x}, T, X, n, r0, kb, j0, flag);
}

// C[i][j] -= sum_q A[i][k0 + q] * B[k0 + q][j] over q < kb, for rows
// [i0, i1) and columns [j0, n) of the n x n row-major C (A, B and C may be
// the same matrix: the rows and columns read are not the ones written).
// Tiles of GM x GM outputs, one per block, 4 x 4 per thread.
VX_DEVK void k_gemm_sub_body(VxBlkB<GT, 0> vb, const double *A, const double *B, double *C, long long n,
                             long long i0, long long i1, long long j0, long long k0, int kb, const int *flag) {
    __shared__ double sa[LU_B][GM + 1];   // A tile, transposed: [q][row]
    __shared__ double sb[LU_B][GM];       // B tile: [q][col]
    if (*flag) return;
    const long long rows = i1 - i0, cols = n - j0;
    const long long tr = (rows + GM - 1) / GM, tc = (cols + GM - 1) / GM;
    const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
    for (long long tile = vb.x; tile < tr * tc; tile += vb.n) {
        const long long bi = i0 + (tile / tc) * GM, bj = j0 + (tile % tc) * GM;
        __syncthreads();
        for (int e = threadIdx.x; e < LU_B * GM; e += blockDim.x) {
            const int r = e / LU_B, q = e % LU_B;            // A: GM rows x LU_B
            const long long gi = bi + r;
            sa[q][r] = (q < kb && gi < i1) ? A[gi * n + k0 + q] : 0.0;
            const int q2 = e / GM, c = e % GM;               // B: LU_B rows x GM
            const long long gj = bj + c;
            sb[q2][c] = (q2 < kb && gj < n) ? B[(k0 + q2) * n + gj] : 0.0;
        }
        __syncthreads();
        double acc[4][4] = {};
#pragma unroll 8
        for (int q = 0; q < LU_B; ++q) {
            double a[4], b[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) a[u] = sa[q][ty * 4 + u];
#pragma unroll
            for (int u = 0; u < 4; ++u) b[u] = sb[q][tx * 4 + u];
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int w = 0; w < 4; ++w) acc[u][w] = fma(a[u], b[w], acc[u][w]);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const long long gi = bi + ty * 4 + u;
            if (gi >= i1) continue;
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                const long long gj = bj + tx * 4 + w;
                if (gj < n) C[gi * n + gj] -= acc[u][w];
            }
        }
    }
}
__global__ void __launch_bounds__(GT) k_gemm_sub(const double *A, const double *B, double *C, long long n,
                                                 long long i0, long long i1, long long j0, long long k0, int kb,
                                                 const int *flag) {
    VX_PDL_WAIT();
    k_gemm_sub_body(VxBlkB<GT, 0>{blockIdx.x, gridDim.x}, A, B, C, n, i0, i1, j0, k0, kb, flag);
}

// X = the row permutation of the identity given by the swaps piv[0..n).
VX_DEVK void k_lu_perm_body(VxBlk vb, double *X, long long n, const int *piv, const int *flag) {
    if (*flag) return;
    for (long long j = vb.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)vb.n * blockDim.x) {
        // column j of P I: e_j with the swaps applied in order
        long long pos = j;
        for (long long r = 0; r < n; ++r) {
            const long long p = piv[r];
            if (pos == r) pos = p;
            else if (pos == p) pos = r;
        }
        for (long long i = 0; i < n; ++i) X[i * n + j] = i == pos ? 1.0 : 0.0;
    }
}
__global__ void k_lu_perm(double *X, long long n, const int *piv, const int *flag) {
    VX_PDL_WAIT();
    k_lu_perm_body(VxBlk{blockIdx.x, gridDim.x}, X, n, piv, flag);
}

// A (n x n, destroyed: it holds L and U afterwards) -> Inv = A^-1.  piv:
// n ints of scratch.
cudaError_t vx_invert_lu(const VxLaunch &L, double *A, double *Inv, long long n, int *piv, int *flag) {
    const int grid = L.num_sms * 4;
    for (long long k0 = 0; k0 < n; k0 += LU_B) {
        const int kb = (int)std::min<long long>(LU_B, n - k0);
        vx_launch<k_lu_panel, k_lu_panel_body>(L, 1, LU_T, 0, A, n, k0, kb, piv, flag);
        vx_launch<k_lu_swap, k_lu_swap_body>(L, (int)vx_ceil_div(n, 256), 256, 0, A, n, k0, kb, (const int *)piv,
                                             (const int *)flag);
        const long long j1 = k0 + kb;
        if (j1 < n) {
            vx_launch<k_lu_trsm<true>, k_lu_trsm_body<true>>(L, (int)std::min<long long>(grid, vx_ceil_div(n - j1, 256)),
                                                             256, 0, (const double *)A, A, n, k0, kb, j1,
                                                             (const int *)flag);
            const long long tiles = vx_ceil_div(n - j1, GM) * vx_ceil_div(n - j1, GM);
            vx_launch<k_gemm_sub, k_gemm_sub_body>(L, (int)std::min<long long>(grid * 2, tiles), GT, 0,
                                                   (const double *)A, (const double *)A, A, n, j1, n, j1, k0, kb,
                                                   (const int *)flag);
        }
    }
    // forward: Inv = L^-1 P
    vx_launch<k_lu_perm, k_lu_perm_body>(L, (int)vx_ceil_div(n, 128), 128, 0, Inv, n, (const int *)piv, (const int *)flag);
    for (long long k0 = 0; k0 < n; k0 += LU_B) {
        const int kb = (int)std::min<long long>(LU_B, n - k0);
        vx_launch<k_lu_trsm<true>, k_lu_trsm_body<true>>(L, (int)std::min<long long>(grid, vx_ceil_div(n, 256)), 256, 0,
                                                         (const double *)A, Inv, n, k0, kb, 0LL, (const int *)flag);
        if (k0 + kb < n) {
            const long long tiles = vx_ceil_div(n - k0 - kb, GM) * vx_ceil_div(n, GM);
            vx_launch<k_gemm_sub, k_gemm_sub_body>(L, (int)std::min<long long>(grid * 2, tiles), GT, 0,
                                                   (const double *)A, (const double *)Inv, Inv, n, k0 + kb, n, 0LL,
                                                   k0, kb, (const int *)flag);
        }
    }
    // backward: Inv = U^-1 Inv
    for (long long k0 = ((n - 1) / LU_B) * LU_B; k0 >= 0; k0 -= LU_B) {
        const int kb = (int)std::min<long long>(LU_B, n - k0);
        vx_launch<k_lu_trsm<false>, k_lu_trsm_body<false>>(L, (int)std::min<long long>(grid, vx_ceil_div(n, 256)), 256,
                                                           0, (const double *)A, Inv, n, k0, kb, 0LL,
                                                           (const int *)flag);
        if (k0 > 0) {
            const long long tiles = vx_ceil_div(k0, GM) * vx_ceil_div(n, GM);
            vx_launch<k_gemm_sub, k_gemm_sub_body>(L, (int)std::min<long long>(grid * 2, tiles), GT, 0,
                                                   (const double *)A, (const double *)Inv, Inv, n, 0LL, k0, 0LL, k0,
                                                   kb, (const int *)flag);
        }
    }
    return cudaGetLastError();
}
