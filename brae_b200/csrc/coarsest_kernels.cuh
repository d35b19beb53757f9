// coarsest_kernels.cuh -- the coarsest-level solve: PCG with DIC from the psi handed in, to the
// preconditioner entry's tolerance and relTol, maxIter 1000 (gamg_solver_cpp.cu:321-383), in ONE
// warp. The coarsest level has nCellsInCoarsestLevel..2x cells (10-20 by default), so the whole
// solve is a few thousand dependent operations: it stays on the device (the reference's device arm
// copies it to the host and back every V-cycle, device_gamg_solver.cu:549-569). Sums and the DIC
// substitution run serially on lane 0 in the reference's order (they decide the iteration count);
// element-wise work is spread over the lanes. Scratch lives in global memory (L1-resident).
// Vectors and rows are in the level's position order; the serial sums and the DIC passes walk cells
// and faces in the reference's order through posOf (cell -> position).
#pragma once

#include "b2g_common.cuh"

namespace b2g {
namespace k {

struct DevPerf
{
    double initialResidual;
    double finalResidual;
    int nIterations;
    int pad;
};

template <class T>
struct CoarsestArgs
{
    int n, nF;
    const int* __restrict__ lower;   // by face, cell ids
    const int* __restrict__ upper;
    const int* __restrict__ posOf;   // cell -> position
    const int* __restrict__ rowStart;  // rows by position (ldu_kernels.cuh Rows)
    const int* __restrict__ col;
    const T* __restrict__ val;
    const T* __restrict__ diag;      // by position
    const T* __restrict__ coef;      // LDU upper, by face
    const T* source;
    T* psi;
    T* pA;
    T* wA;
    T* rA;
    T* rD;
    T tolerance;
    T relTol;
    int maxIter;
    DevPerf* log;       // may be null
    int* logCount;      // appended when log != null
    int logCapacity;
    DevPerf* out;       // may be null
    // the level's coupled pair by position (ldu_kernels.cuh Rows), or null: Amul subtracts
    // pairVal * x[pairCol] after the face terms, sumA subtracts pairVal (GAMG:82-87, :137-145); DIC's
    // factorisation does not see it (GAMG:194-231)
    const int* __restrict__ pairStart = nullptr;
    const int* __restrict__ pairCol = nullptr;
    const T* __restrict__ pairVal = nullptr;
};

template <class T> struct PerfConst;
template <> struct PerfConst<double>
{
    static constexpr double small = 1e-20, vsmall = 1e-300, great = 1e+20;
};
template <> struct PerfConst<float>
{
    static constexpr float small = 1e-20f, vsmall = 1e-37f, great = 1e+20f;
};

template <class T>
__device__ __forceinline__ void warpAmul(const CoarsestArgs<T>& a, const T* x, T* y)
{
    for (int c = threadIdx.x; c < a.n; c += 32)
    {
        T acc = mulRn(a.diag[c], x[c]);
        for (int e = a.rowStart[c]; e < a.rowStart[c + 1]; ++e) acc = addRn(acc, mulRn(a.val[e], x[a.col[e]]));
        if (a.pairStart)
            for (int k = a.pairStart[c]; k < a.pairStart[c + 1]; ++k)
                acc = subRn(acc, mulRn(a.pairVal[k], x[a.pairCol[k]]));
        y[c] = acc;
    }
    __syncwarp();
}

template <class T>
__device__ __forceinline__ T serialSumProd(int n, const int* posOf, const T* x, const T* y)
{
    T s = T(0);
    for (int c = 0; c < n; ++c) s = addRn(s, mulRn(x[posOf[c]], y[posOf[c]]));
    return s;
}

template <class T>
__device__ __forceinline__ T serialSumMag(int n, const int* posOf, const T* x)
{
    T s = T(0);
    for (int c = 0; c < n; ++c) s = addRn(s, fabs(x[posOf[c]]));
    return s;
}

template <class T>
__device__ __forceinline__ bool convergedT(T fin, T init, T tol, T relTol)
{
    return fin < tol || (relTol > PerfConst<T>::small && fin < mulRn(relTol, init));
}

// One warp (blockDim.x == 32).
template <class T>
__device__ __forceinline__ void coarsestPcgDicWarp(const CoarsestArgs<T>& a)
{
    __shared__ T shScal[4];  // nf, init, final, flag
    __shared__ int shIter;
    __shared__ int shStop;
    const int lane = threadIdx.x;
    const int n = a.n;
    warpAmul(a, a.psi, a.wA);
    for (int c = lane; c < n; c += 32) a.rA[c] = subRn(a.source[c], a.wA[c]);
    // normFactor's row sums into pA (scratch, as the reference uses it)
    for (int c = lane; c < n; c += 32)
    {
        T s = a.diag[c];
        for (int e = a.rowStart[c]; e < a.rowStart[c + 1]; ++e) s = addRn(s, a.val[e]);
        if (a.pairStart)
            for (int k = a.pairStart[c]; k < a.pairStart[c + 1]; ++k) s = subRn(s, a.pairVal[k]);
        a.pA[c] = s;
    }
    __syncwarp();
    if (lane == 0)
    {
        const int* po = a.posOf;
        T avg = T(0);
        for (int c = 0; c < n; ++c) avg = addRn(avg, a.psi[po[c]]);
        avg = divRn(avg, static_cast<T>(n));
        T sum = T(0);
        for (int c = 0; c < n; ++c)
        {
            const int i = po[c];
            const T t = mulRn(a.pA[i], avg);
            sum = addRn(sum, addRn(fabs(subRn(a.wA[i], t)), fabs(subRn(a.source[i], t))));
        }
        const T nf = addRn(sum, PerfConst<T>::small);
        const T init = divRn(serialSumMag(n, po, a.rA), nf);
        shScal[0] = nf;
        shScal[1] = init;
        shScal[2] = init;
        shIter = 0;
        shStop = convergedT(init, init, a.tolerance, a.relTol) ? 1 : 0;
        if (!shStop)
        {
            // DICPreconditioner::calcReciprocalD (GAMG:194-210)
            for (int i = 0; i < n; ++i) a.rD[i] = a.diag[i];
            for (int f = 0; f < a.nF; ++f)
            {
                const int u = po[a.upper[f]];
                a.rD[u] = subRn(a.rD[u], divRn(mulRn(a.coef[f], a.coef[f]), a.rD[po[a.lower[f]]]));
            }
            for (int i = 0; i < n; ++i) a.rD[i] = divRn(T(1), a.rD[i]);
        }
    }
    __syncwarp();
    __syncthreads();
    T wArA = PerfConst<T>::great;
    const T nf = shScal[0];
    while (!shStop)
    {
        const T wArAold = wArA;
        for (int c = lane; c < n; c += 32) a.wA[c] = mulRn(a.rD[c], a.rA[c]);
        __syncwarp();
        if (lane == 0)
        {
            // the two DIC substitution passes (GAMG:212-231)
            const int* po = a.posOf;
            for (int f = 0; f < a.nF; ++f)
            {
                const int u = po[a.upper[f]];
                a.wA[u] = subRn(a.wA[u], mulRn(mulRn(a.rD[u], a.coef[f]), a.wA[po[a.lower[f]]]));
            }
            for (int f = a.nF - 1; f >= 0; --f)
            {
                const int l = po[a.lower[f]];
                a.wA[l] = subRn(a.wA[l], mulRn(mulRn(a.rD[l], a.coef[f]), a.wA[po[a.upper[f]]]));
            }
            shScal[3] = serialSumProd(n, po, a.wA, a.rA);
        }
        __syncthreads();
        wArA = shScal[3];
        if (shIter == 0)
        {
            for (int c = lane; c < n; c += 32) a.pA[c] = a.wA[c];
        }
        else
        {
            const T beta = divRn(wArA, wArAold);
            for (int c = lane; c < n; c += 32) a.pA[c] = addRn(a.wA[c], mulRn(beta, a.pA[c]));
        }
        __syncwarp();
        warpAmul(a, a.pA, a.wA);
        if (lane == 0) shScal[3] = serialSumProd(n, a.posOf, a.wA, a.pA);
        __syncthreads();
        const T wApA = shScal[3];
        if (divRn(fabs(wApA), nf) < PerfConst<T>::vsmall) break;  // checkSingularity
        const T alpha = divRn(wArA, wApA);
        for (int c = lane; c < n; c += 32)
        {
            a.psi[c] = addRn(a.psi[c], mulRn(alpha, a.pA[c]));
            a.rA[c] = subRn(a.rA[c], mulRn(alpha, a.wA[c]));
        }
        __syncwarp();
        if (lane == 0)
        {
            shScal[2] = divRn(serialSumMag(n, a.posOf, a.rA), nf);
            ++shIter;
            shStop = (shIter >= a.maxIter || convergedT(shScal[2], shScal[1], a.tolerance, a.relTol)) ? 1 : 0;
        }
        __syncthreads();
    }
    if (lane == 0)
    {
        DevPerf p;
        p.initialResidual = static_cast<double>(shScal[1]);
        p.finalResidual = static_cast<double>(shScal[2]);
        p.nIterations = shIter;
        p.pad = 0;
        if (a.out) *a.out = p;
        if (a.log)
        {
            const int i = *a.logCount;
            if (i < a.logCapacity) a.log[i] = p;
            *a.logCount = i + 1;
        }
    }
}

template <class T>
__global__ void __launch_bounds__(32) coarsestPcgDic(CoarsestArgs<T> a)
{
    coarsestPcgDicWarp<T>(a);
}

// The coarsest solves of many independent cases, one warp each (block i solves cases[i]) to the
// given tolerance and relTol; a case whose `active` flag (may be null) is 0 is skipped.
static __global__ void __launch_bounds__(32) coarsestPcgDicBatch(const CoarsestArgs<double>* __restrict__ cases,
                                                          double tolerance, double relTol,
                                                          const int* __restrict__ active)
{
    if (active && active[blockIdx.x] == 0) return;
    CoarsestArgs<double> a = cases[blockIdx.x];
    a.tolerance = tolerance;
    a.relTol = relTol;
    coarsestPcgDicWarp<double>(a);
}

// ---------------------------------------------------------------------------------------------
// The coarsest level solved directly, for the FP32-preconditioned forms: a dense FP64 Cholesky
// factor A = L L^T, made once per coarse matrix and applied by two triangular substitutions in
// every V-cycle (the reference's precision/serving form solves its coarsest level directly too,
// device_amg_coarse.cu:545-700; the FP64 parity form keeps the reference's PCG-DIC). The level is
// numbered by position, as its vectors are. The factor is taken only when every pivot is above
// kDensePivotMin * max|diag| (a singular, all-Neumann level is left to PCG-DIC).
// ---------------------------------------------------------------------------------------------

constexpr int kDenseMax = 96;              // the largest coarsest level factored densely
constexpr int kDenseRows = kDenseMax / 32; // rows a lane holds in the substitutions
constexpr double kDensePivotMin = 1e-10;

struct DenseArgs
{
    int n, nF;
    const int* __restrict__ lower;   // by face, cell ids
    const int* __restrict__ upper;
    const int* __restrict__ posOf;   // cell -> position
    const double* __restrict__ diag; // by position
    const double* __restrict__ coef; // by face
    double* L;                       // [n * n] column-major: L(i, k) at k * n + i (lower triangle)
    int* ok;                         // 1: L holds the factor; 0: a pivot was too small
};

// One warp: A into shared memory (column-major, both triangles), then right-looking Cholesky one
// column at a time -- the pivot's square root, the column divided by it, the trailing lower
// triangle updated by the column's outer product. Each entry is updated in increasing k, so the
// factor does not depend on how lanes share the work. Shared memory: n * n doubles.
static __global__ void __launch_bounds__(32) coarseDenseFactor(DenseArgs a)
{
    extern __shared__ double denseSh[];
    const int n = a.n;
    const int lane = threadIdx.x;
    for (int i = lane; i < n * n; i += 32) denseSh[i] = 0.0;
    __syncwarp();
    double dmax = 0.0;
    for (int c = lane; c < n; c += 32)
    {
        const double d = a.diag[c];
        denseSh[c * n + c] = d;
        dmax = fmax(dmax, fabs(d));
    }
    for (int f = lane; f < a.nF; f += 32)
    {
        const int pl = a.posOf[a.lower[f]], pu = a.posOf[a.upper[f]];
        denseSh[pl * n + pu] = a.coef[f];
        denseSh[pu * n + pl] = a.coef[f];
    }
    for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    __syncwarp();
    int ok = 1;
    for (int k = 0; k < n && ok; ++k)
    {
        const double d = denseSh[k * n + k];
        if (!(d > kDensePivotMin * dmax))
        {
            ok = 0;
            break;
        }
        const double lkk = sqrt(d);
        __syncwarp();
        for (int i = k + 1 + lane; i < n; i += 32) denseSh[k * n + i] = divRn(denseSh[k * n + i], lkk);
        if (lane == 0) denseSh[k * n + k] = lkk;
        __syncwarp();
        const int m = n - k - 1;
        for (int idx = lane; idx < m * m; idx += 32)
        {
            const int jj = idx / m, ii = idx % m;
            if (ii < jj) continue;
            const int i = k + 1 + ii, j = k + 1 + jj;
            denseSh[j * n + i] = subRn(denseSh[j * n + i], mulRn(denseSh[k * n + i], denseSh[k * n + j]));
        }
        __syncwarp();
    }
    for (int i = lane; i < n * n; i += 32) a.L[i] = denseSh[i];
    if (lane == 0) *a.ok = ok;
}

// x = L^-T L^-1 b by one warp: row i in lane i % 32, slot i / 32 (registers); the factor in shared
// memory. Forward: y_k /= L(k,k), then y_i -= L(i,k) y_k below it; backward with L^T the same
// upwards. b and x by position, in T (widened to FP64 and narrowed back).
template <class T>
__device__ __forceinline__ void denseSolveWarp(int n, const double* __restrict__ L, const T* __restrict__ b,
                                               T* __restrict__ x, double* sh)
{
    const int lane = threadIdx.x;
    for (int i = lane; i < n * n; i += 32) sh[i] = L[i];
    double y[kDenseRows];
#pragma unroll
    for (int s = 0; s < kDenseRows; ++s)
    {
        const int i = lane + 32 * s;
        y[s] = i < n ? static_cast<double>(b[i]) : 0.0;
    }
    __syncwarp();
    for (int k = 0; k < n; ++k)
    {
        const int ks = k >> 5;
#pragma unroll
        for (int s = 0; s < kDenseRows; ++s)
            if (s == ks && (k & 31) == lane) y[s] = divRn(y[s], sh[k * n + k]);
        double v = 0.0;
#pragma unroll
        for (int s = 0; s < kDenseRows; ++s)
            if (s == ks) v = y[s];
        const double yk = __shfl_sync(0xffffffffu, v, k & 31);
#pragma unroll
        for (int s = 0; s < kDenseRows; ++s)
        {
            const int i = lane + 32 * s;
            if (i > k && i < n) y[s] = subRn(y[s], mulRn(sh[k * n + i], yk));
        }
    }
    for (int k = n - 1; k >= 0; --k)
    {
        const int ks = k >> 5;
#pragma unroll
        for (int s = 0; s < kDenseRows; ++s)
            if (s == ks && (k & 31) == lane) y[s] = divRn(y[s], sh[k * n + k]);
        double v = 0.0;
#pragma unroll
        for (int s = 0; s < kDenseRows; ++s)
            if (s == ks) v = y[s];
        const double yk = __shfl_sync(0xffffffffu, v, k & 31);
#pragma unroll
        for (int s = 0; s < kDenseRows; ++s)
        {
            const int i = lane + 32 * s;
            if (i < k) y[s] = subRn(y[s], mulRn(sh[i * n + k], yk));
        }
    }
#pragma unroll
    for (int s = 0; s < kDenseRows; ++s)
    {
        const int i = lane + 32 * s;
        if (i < n) x[i] = static_cast<T>(y[s]);
    }
}

template <class T>
__global__ void __launch_bounds__(32) coarseDenseSolve(int n, const double* __restrict__ L, const T* __restrict__ b,
                                                       T* __restrict__ x)
{
    extern __shared__ double denseSh[];
    denseSolveWarp<T>(n, L, b, x, denseSh);
}

// Many cases' coarsest levels, one warp each (block i: case i), skipped where `active` is 0 or the
// case has no factor (n = 0).
struct DenseCase
{
    int n;
    const double* L;
    const float* b;
    float* x;
};
static __global__ void __launch_bounds__(32) coarseDenseSolveBatch(const DenseCase* __restrict__ cases,
                                                                  const int* __restrict__ active)
{
    extern __shared__ double denseSh[];
    if (active && active[blockIdx.x] == 0) return;
    const DenseCase c = cases[blockIdx.x];
    if (c.n == 0) return;
    denseSolveWarp<float>(c.n, c.L, c.b, c.x, denseSh);
}

}  // namespace k
}  // namespace b2g
