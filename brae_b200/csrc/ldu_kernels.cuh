// ldu_kernels.cuh -- the LDU kernels of one level, templated on the value type (double for the
// parity form, float for the FP32 V-cycle). Every kernel walks a cell's terms in the reference's
// accumulation order with separately rounded products and sums, so the FP64 instances are
// bit-for-bit the reference's host loops.
//
// Reference: GAMG = src/matrices/lduMatrix/solvers/GAMG/gamg_solver_cpp.cu
#pragma once

#include "b2g_common.cuh"

namespace b2g {
namespace k {

template <class T> struct Small;
template <> struct Small<double>
{
    static constexpr double vsmall = 1e-300;  // solverPerformance::vsmall_ (GAMG:17)
};
template <> struct Small<float>
{
    static constexpr float vsmall = 1e-37f;
};

// Rows of one level, in the level's position (sweep) order: for the cell at position i the entries
// [rowStart[i], rowStart[i+1]) hold first the faces the cell is the neighbour of, then the faces it
// owns, each ascending -- the order in which lduMatrix::Amul and lduMatrix::residual add a cell's
// terms (GAMG:62-117). `col` is the other cell's position, `val` the coefficient per entry, `diag`
// the diagonal by position. Every per-cell result is the reference's bit for bit; only where the
// cells sit in memory differs.
//
// A coupled (cyclic) pair, when the level carries one (pair.cu): per position the pair faces the cell
// owns, in face order -- [pairStart[i], pairStart[i+1]) -- with the neighbour's position and the
// coefficient, in the reference's sign convention (Amul subtracts coefficient * x[neighbour],
// GAMG:82-87). pairStart null: no pair, and every kernel below computes exactly what it did without.
template <class T>
struct Rows
{
    int n;
    const int* __restrict__ rowStart;
    const int* __restrict__ col;
    const T* __restrict__ val;
    const T* __restrict__ diag;
    const int* __restrict__ pairStart = nullptr;
    const int* __restrict__ pairCol = nullptr;
    const T* __restrict__ pairVal = nullptr;
    // the same rows in sliced ELL, where the level has it: the row of position c is lane c % 32 of
    // slice c / 32, its entry q at ellBase[slice] + 32*q + lane (column -1 past the row's end), so a
    // warp's 32 rows load each entry in one coalesced access
    const int* __restrict__ ellBase = nullptr;
    const int* __restrict__ ellCol = nullptr;
    const T* __restrict__ ellVal = nullptr;
};

// The row of position c folded into acc in the row's entry order: acc = term(acc, coefficient, column
// position) per entry, from the sliced ELL copy when the level has one, else from the CSR rows -- the
// same entries in the same order either way.
template <class T, class F>
__device__ __forceinline__ T rowFold(const Rows<T>& A, int c, T acc, F term)
{
    if (A.ellBase)
    {
        const int sl = c >> 5, lane = c & 31;
        const int b0 = A.ellBase[sl];
        const int w = (A.ellBase[sl + 1] - b0) >> 5;
        // no early exit: the padding entries (column -1) are all past the row's end and skipped,
        // and without a data-dependent branch the loads of several entries are in flight at once
#pragma unroll 4
        for (int q = 0; q < w; ++q)
        {
            const int e = b0 + 32 * q + lane;
            const int cp = A.ellCol[e];
            const T v = A.ellVal[e];
            if (cp >= 0) acc = term(acc, v, cp);
        }
        return acc;
    }
    const int e1 = A.rowStart[c + 1];
    for (int e = A.rowStart[c]; e < e1; ++e) acc = term(acc, A.val[e], A.col[e]);
    return acc;
}

// The pair's terms of row c after the face terms, in face order: acc - coef*x[nbr] each (Amul's sign)
template <class T>
__device__ __forceinline__ T pairSub(const Rows<T>& A, int c, T acc, const T* __restrict__ x)
{
    if (A.pairStart)
    {
        const int k1 = A.pairStart[c + 1];
        for (int k = A.pairStart[c]; k < k1; ++k) acc = subRn(acc, mulRn(A.pairVal[k], x[A.pairCol[k]]));
    }
    return acc;
}

// lduMatrix::Amul (GAMG:62-88): y = diag*x, then the face terms in face order
template <class T>
__global__ void amul(Rows<T> A, const T* __restrict__ x, T* __restrict__ y)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < A.n; c += gridDim.x * blockDim.x)
    {
        T acc = mulRn(A.diag[c], x[c]);
        acc = rowFold(A, c, acc, [x](T a, T v, int cp) { return addRn(a, mulRn(v, x[cp])); });
        y[c] = pairSub(A, c, acc, x);
    }
}

// A block-wide sum in a fixed shape (deterministic for a fixed blockDim).
template <class T, int NT>
__device__ __forceinline__ T blockSum(T v, T* sh)
{
    for (int o = 16; o > 0; o >>= 1) v = addRn(v, __shfl_down_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) sh[w] = v;
    __syncthreads();
    T r = T(0);
    if (threadIdx.x < 32)
    {
        r = threadIdx.x < NT / 32 ? sh[threadIdx.x] : T(0);
        for (int o = 16; o > 0; o >>= 1) r = addRn(r, __shfl_down_sync(0xffffffffu, r, o));
    }
    __syncthreads();
    return r;  // valid in thread 0
}

// GAMGSolver::scale, first half (GAMG:391-399): Acf = A*field and per-block partial sums of
// field.source and field.Acf (sums in a fixed tree; the reference sums serially, so these agree to
// rounding, not bitwise).
template <class T, int NT>
__global__ void __launch_bounds__(NT) amulScaleDots(Rows<T> A, const T* __restrict__ field,
                                                    const T* __restrict__ source, T* __restrict__ Acf,
                                                    T* __restrict__ partial)
{
    __shared__ T sh[NT / 32];
    T num = T(0), den = T(0);
    for (int c = blockIdx.x * NT + threadIdx.x; c < A.n; c += gridDim.x * NT)
    {
        const T fc = field[c];
        T acc = mulRn(A.diag[c], fc);
        acc = rowFold(A, c, acc, [field](T a, T v, int cp) { return addRn(a, mulRn(v, field[cp])); });
        acc = pairSub(A, c, acc, field);
        Acf[c] = acc;
        num = addRn(num, mulRn(fc, source[c]));
        den = addRn(den, mulRn(fc, acc));
    }
    num = blockSum<T, NT>(num, sh);
    den = blockSum<T, NT>(den, sh);
    if (threadIdx.x == 0)
    {
        partial[2 * blockIdx.x] = num;
        partial[2 * blockIdx.x + 1] = den;
    }
}

// sf = (x.b)/stabilise(x.Ax, vsmall) (GAMG:400-401) from the partials, in one block
template <class T, int NT>
__global__ void __launch_bounds__(NT) scaleFactor(const T* __restrict__ partial, int nPartial, T* __restrict__ sf)
{
    __shared__ T sh[NT / 32];
    T num = T(0), den = T(0);
    for (int i = threadIdx.x; i < nPartial; i += NT)
    {
        num = addRn(num, partial[2 * i]);
        den = addRn(den, partial[2 * i + 1]);
    }
    num = blockSum<T, NT>(num, sh);
    den = blockSum<T, NT>(den, sh);
    if (threadIdx.x == 0)
    {
        const T v = Small<T>::vsmall;
        *sf = divRn(num, den >= T(0) ? addRn(den, v) : subRn(den, v));
    }
}

// field = sf*field + (source - sf*Acf)/diag (GAMG:402-406)
template <class T>
__global__ void scaleUpdate(int n, const T* __restrict__ sfp, T* __restrict__ field, const T* __restrict__ source,
                            const T* __restrict__ Acf, const T* __restrict__ diag)
{
    const T sf = *sfp;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    {
        field[c] = addRn(mulRn(sf, field[c]), divRn(subRn(source[c], mulRn(sf, Acf[c])), diag[c]));
    }
}

// The finest level's scale update fused with psi += finestCorrection (GAMG:716-723): the
// correction is formed exactly as scale() forms it and added exactly as the reference adds it.
template <class T>
__global__ void scaleUpdateAdd(int n, const T* __restrict__ sfp, const T* __restrict__ field,
                               const T* __restrict__ source, const T* __restrict__ Acf, const T* __restrict__ diag,
                               T* __restrict__ psi)
{
    const T sf = *sfp;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    {
        const T corr = addRn(mulRn(sf, field[c]), divRn(subRn(source[c], mulRn(sf, Acf[c])), diag[c]));
        psi[c] = addRn(psi[c], corr);
    }
}

// THE FINEST LEVEL'S CORRECTION, FUSED: prolongField (GAMG:422-432) injects the coarse correction
// into a fine vector that only the scaling and the update then read. Here that vector is never
// stored: every read of it takes coarse[prolongP[c]] instead -- the same values, the same operations in
// the same order, so the results are those of the three separate steps bit for bit. (Not for a level
// with a coupled pair, whose Amul reads the pair's neighbours too.)
template <class T, int NT>
__global__ void __launch_bounds__(NT) amulScaleDotsProlong(Rows<T> A, const int* __restrict__ prolongP,
                                                           const int* __restrict__ ellColCoarse,
                                                           const T* __restrict__ coarse,
                                                           const T* __restrict__ source, T* __restrict__ Acf,
                                                           T* __restrict__ partial)
{
    __shared__ T sh[NT / 32];
    T num = T(0), den = T(0);
    for (int c = blockIdx.x * NT + threadIdx.x; c < A.n; c += gridDim.x * NT)
    {
        const T fc = coarse[prolongP[c]];
        T acc = mulRn(A.diag[c], fc);
        if (A.ellBase && ellColCoarse)
        {
            // the sliced rows with each column's coarse position at hand: one gather per entry
            const int sl = c >> 5, lane = c & 31;
            const int b0 = A.ellBase[sl];
            const int w = (A.ellBase[sl + 1] - b0) >> 5;
#pragma unroll 4
            for (int q = 0; q < w; ++q)
            {
                const int e = b0 + 32 * q + lane;
                const int cc = ellColCoarse[e];
                const T v = A.ellVal[e];
                if (cc >= 0) acc = addRn(acc, mulRn(v, coarse[cc]));
            }
        }
        else
        {
            acc = rowFold(A, c, acc,
                          [coarse, prolongP](T a, T v, int cp) { return addRn(a, mulRn(v, coarse[prolongP[cp]])); });
        }
        Acf[c] = acc;
        num = addRn(num, mulRn(fc, source[c]));
        den = addRn(den, mulRn(fc, acc));
    }
    num = blockSum<T, NT>(num, sh);
    den = blockSum<T, NT>(den, sh);
    if (threadIdx.x == 0)
    {
        partial[2 * blockIdx.x] = num;
        partial[2 * blockIdx.x + 1] = den;
    }
}

// psi += sf*P + (source - sf*Acf)/diag with P = coarse[prolongP[c]] (scaleUpdateAdd on the injection)
template <class T>
__global__ void scaleUpdateAddProlong(int n, const T* __restrict__ sfp, const int* __restrict__ prolongP,
                                      const T* __restrict__ coarse, const T* __restrict__ source,
                                      const T* __restrict__ Acf, const T* __restrict__ diag, T* __restrict__ psi)
{
    const T sf = *sfp;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    {
        const T corr = addRn(mulRn(sf, coarse[prolongP[c]]), divRn(subRn(source[c], mulRn(sf, Acf[c])), diag[c]));
        psi[c] = addRn(psi[c], corr);
    }
}

// The residual between V-cycles, FUSED: Apsi = A*psi (Amul's order) and r = source - Apsi in one pass,
// the product never stored (Amul then subtract, bit for bit)
template <class T>
__global__ void amulSubtract(Rows<T> A, const T* __restrict__ source, const T* __restrict__ x, T* __restrict__ r)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < A.n; c += gridDim.x * blockDim.x)
    {
        T acc = mulRn(A.diag[c], x[c]);
        acc = rowFold(A, c, acc, [x](T a, T v, int cp) { return addRn(a, mulRn(v, x[cp])); });
        r[c] = subRn(source[c], pairSub(A, c, acc, x));
    }
}

// psi += correction, unscaled (scaleCorrection off)
template <class T>
__global__ void addInPlace(int n, T* __restrict__ psi, const T* __restrict__ corr)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        psi[c] = addRn(psi[c], corr[c]);
}

// restrictField (GAMG:410-419): cf = 0; cf[map[i]] += ff[i] for ascending i -- gathered per coarse
// cell over its fine cells in ascending fine-cell order (lists of positions on both levels)
template <class T>
__global__ void restrictField(int nCoarse, const int* __restrict__ cellStart, const int* __restrict__ cellList,
                              const T* __restrict__ ff, T* __restrict__ cf)
{
    for (int C = blockIdx.x * blockDim.x + threadIdx.x; C < nCoarse; C += gridDim.x * blockDim.x)
    {
        T acc = T(0);
        const int e1 = cellStart[C + 1];
        for (int e = cellStart[C]; e < e1; ++e) acc = addRn(acc, ff[cellList[e]]);
        cf[C] = acc;
    }
}

// prolongField (GAMG:422-432): injection, overwriting
template <class T>
__global__ void prolongField(int nFine, const int* __restrict__ map, const T* __restrict__ cf, T* __restrict__ ff)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nFine; i += gridDim.x * blockDim.x)
        ff[i] = cf[map[i]];
}

// agglomerateMatrix (GAMG:474-496), diagonal: restrictField of the fine diagonal, then
// 2*upper of every fine face inside the coarse cell, ascending
static __global__ void galerkinDiag(int nCoarse, const int* __restrict__ cellStart, const int* __restrict__ cellList,
                             const int* __restrict__ intStart, const int* __restrict__ intList,
                             const double* __restrict__ fdiag, const double* __restrict__ fupper,
                             double* __restrict__ cdiag)
{
    for (int C = blockIdx.x * blockDim.x + threadIdx.x; C < nCoarse; C += gridDim.x * blockDim.x)
    {
        double acc = 0.0;
        for (int e = cellStart[C]; e < cellStart[C + 1]; ++e) acc = __dadd_rn(acc, fdiag[cellList[e]]);
        for (int e = intStart[C]; e < intStart[C + 1]; ++e) acc = __dadd_rn(acc, __dmul_rn(2.0, fupper[intList[e]]));
        cdiag[C] = acc;
    }
}

// agglomerateMatrix, coarse upper: the sum of its fine faces' coefficients, ascending
static __global__ void galerkinUpper(int nCF, const int* __restrict__ faceBeg, const int* __restrict__ faceEnd,
                              const int* __restrict__ faceList, const double* __restrict__ fupper,
                              double* __restrict__ cupper)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nCF; p += gridDim.x * blockDim.x)
    {
        double acc = 0.0;
        for (int e = faceBeg[p]; e < faceEnd[p]; ++e) acc = __dadd_rn(acc, fupper[faceList[e]]);
        cupper[p] = acc;
    }
}

// the per-entry coefficient of the row layout
template <class T, class S>
__global__ void gatherVal(long long nnz, const int* __restrict__ entFace, const S* __restrict__ upper,
                          T* __restrict__ val)
{
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nnz;
         e += (long long)gridDim.x * blockDim.x)
        val[e] = static_cast<T>(upper[entFace[e]]);
}

template <class T, class S>
__global__ void castArray(long long n, const S* __restrict__ in, T* __restrict__ out)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = static_cast<T>(in[i]);
}

// natural cell order <-> position order: pos[i] = nat[posCell[i]] and back
template <class T>
__global__ void toPositions(int n, const int* __restrict__ posCell, const T* __restrict__ nat, T* __restrict__ pos)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) pos[i] = nat[posCell[i]];
}
template <class T>
__global__ void fromPositions(int n, const int* __restrict__ posCell, const T* __restrict__ pos, T* __restrict__ nat)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) nat[posCell[i]] = pos[i];
}

// lduMatrix::residual (GAMG:90-117): r = source - diag*psi, then minus the face terms in order
template <class T>
__global__ void residual(Rows<T> A, const T* __restrict__ source, const T* __restrict__ psi, T* __restrict__ r)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < A.n; c += gridDim.x * blockDim.x)
    {
        T acc = subRn(source[c], mulRn(A.diag[c], psi[c]));
        acc = rowFold(A, c, acc, [psi](T a, T v, int cp) { return subRn(a, mulRn(v, psi[cp])); });
        // the pair with the sign Amul's term does not have (GAMG:110-115)
        if (A.pairStart)
            for (int k = A.pairStart[c]; k < A.pairStart[c + 1]; ++k)
                acc = addRn(acc, mulRn(A.pairVal[k], psi[A.pairCol[k]]));
        r[c] = acc;
    }
}

// r = a - b
template <class T>
__global__ void subtract(int n, const T* __restrict__ a, const T* __restrict__ b, T* __restrict__ r)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        r[c] = subRn(a[c], b[c]);
}

// Two-stage deterministic reductions into a device slot. Stage one: a fixed grid of NT-thread
// blocks, each thread walking a grid stride; stage two: one block over the partials.
enum ReduceOp : int { RED_DOT = 0, RED_SUMMAG = 1, RED_SUM = 2 };

template <class T, int NT, int OP>
__global__ void __launch_bounds__(NT) reducePartial(int n, const T* __restrict__ a, const T* __restrict__ b,
                                                    T* __restrict__ partial)
{
    __shared__ T sh[NT / 32];
    T s = T(0);
    for (int i = blockIdx.x * NT + threadIdx.x; i < n; i += gridDim.x * NT)
    {
        if (OP == RED_DOT) s = addRn(s, mulRn(a[i], b[i]));
        else if (OP == RED_SUMMAG) s = addRn(s, fabs(a[i]));
        else s = addRn(s, a[i]);
    }
    s = blockSum<T, NT>(s, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

template <class T, int NT>
__global__ void __launch_bounds__(NT) reduceFinal(const T* __restrict__ partial, int nPartial, T* __restrict__ out)
{
    __shared__ T sh[NT / 32];
    T s = T(0);
    for (int i = threadIdx.x; i < nPartial; i += NT) s = addRn(s, partial[i]);
    s = blockSum<T, NT>(s, sh);
    if (threadIdx.x == 0) *out = s;
}

// sumA's pair terms (GAMG:137-145): minus each coefficient, in face order
template <class T>
__device__ __forceinline__ T pairRowSum(const Rows<T>& A, int c, T sumA)
{
    if (A.pairStart)
        for (int k = A.pairStart[c]; k < A.pairStart[c + 1]; ++k) sumA = subRn(sumA, A.pairVal[k]);
    return sumA;
}

// GaussSeidelSmoother's bPrime with the pair moved to the right-hand side (GAMG:287-305): source plus
// coefficient * psi[neighbour] per pair face, in face order, from psi as it stands
template <class T>
__global__ void pairFold(Rows<T> A, const T* __restrict__ source, const T* __restrict__ psi, T* __restrict__ bPrime)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < A.n; c += gridDim.x * blockDim.x)
    {
        T b = source[c];
        for (int k = A.pairStart[c]; k < A.pairStart[c + 1]; ++k) b = addRn(b, mulRn(A.pairVal[k], psi[A.pairCol[k]]));
        bPrime[c] = b;
    }
}

// normFactor (GAMG:119-159), the per-cell summand |Apsi - t| + |source - t| with t = sumA*xRef;
// sumA = diag + the row's coefficients in row order (the reference adds a cell's face terms in
// face order, which is row order)
template <class T, int NT>
__global__ void __launch_bounds__(NT) normFactorPartial(Rows<T> A, const T* __restrict__ psi, const T* __restrict__ source,
                                                        const T* __restrict__ Apsi, const T* __restrict__ sumPsi,
                                                        T* __restrict__ partial)
{
    __shared__ T sh[NT / 32];
    const T xRef = divRn(*sumPsi, static_cast<T>(A.n));
    T s = T(0);
    for (int c = blockIdx.x * NT + threadIdx.x; c < A.n; c += gridDim.x * NT)
    {
        T sumA = A.diag[c];
        const int e1 = A.rowStart[c + 1];
        for (int e = A.rowStart[c]; e < e1; ++e) sumA = addRn(sumA, A.val[e]);
        sumA = pairRowSum(A, c, sumA);
        const T t = mulRn(sumA, xRef);
        s = addRn(s, addRn(fabs(subRn(Apsi[c], t)), fabs(subRn(source[c], t))));
    }
    s = blockSum<T, NT>(s, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// Serial reductions in the reference's order: one warp streams the terms in cell order (the value of
// cell c sits at position posOf[c]), lane 0 adds them one after another (s = ((s + t0) + t1) + ...),
// exactly as the reference's host loops do.
template <int OP>
__global__ void __launch_bounds__(32) serialReduce(int n, const double* __restrict__ a, const double* __restrict__ b,
                                                   const int* __restrict__ posOf, double* __restrict__ out)
{
    const int lane = threadIdx.x;
    double s = 0.0;
    for (int base = 0; base < n; base += 32)
    {
        const int c = base + lane;
        double term = 0.0;
        if (c < n)
        {
            const int i = posOf[c];
            if (OP == RED_DOT) term = __dmul_rn(a[i], b[i]);
            else if (OP == RED_SUMMAG) term = fabs(a[i]);
            else term = a[i];
        }
        const int cnt = min(32, n - base);
        for (int j = 0; j < cnt; ++j)
        {
            const double v = __shfl_sync(0xffffffffu, term, j);
            if (lane == 0) s = __dadd_rn(s, v);
        }
    }
    if (lane == 0) *out = s;
}

// scale's two sums in one serial pass: num += field*source, den += field*Acf
static __global__ void __launch_bounds__(32) serialScaleDots(int n, const double* __restrict__ field,
                                                      const double* __restrict__ source, const double* __restrict__ Acf,
                                                      const int* __restrict__ posOf, double* __restrict__ sf)
{
    const int lane = threadIdx.x;
    double num = 0.0, den = 0.0;
    for (int base = 0; base < n; base += 32)
    {
        const int c = base + lane;
        double tn = 0.0, td = 0.0;
        if (c < n)
        {
            const int i = posOf[c];
            tn = __dmul_rn(field[i], source[i]);
            td = __dmul_rn(field[i], Acf[i]);
        }
        const int cnt = min(32, n - base);
        for (int j = 0; j < cnt; ++j)
        {
            const double vn = __shfl_sync(0xffffffffu, tn, j);
            const double vd = __shfl_sync(0xffffffffu, td, j);
            if (lane == 0)
            {
                num = __dadd_rn(num, vn);
                den = __dadd_rn(den, vd);
            }
        }
    }
    if (lane == 0) *sf = __ddiv_rn(num, den >= 0.0 ? __dadd_rn(den, Small<double>::vsmall) : __dsub_rn(den, Small<double>::vsmall));
}

// normFactor's sum in the reference's order (GAMG:146-157), with sumA from the rows
static __global__ void __launch_bounds__(32) serialNormFactor(Rows<double> A, const double* __restrict__ psi,
                                                       const double* __restrict__ source, const double* __restrict__ Apsi,
                                                       const int* __restrict__ posOf, double* __restrict__ out)
{
    const int lane = threadIdx.x;
    double sumPsi = 0.0;
    for (int base = 0; base < A.n; base += 32)
    {
        const int i = base + lane;
        const double v = i < A.n ? psi[posOf[i]] : 0.0;
        const int cnt = min(32, A.n - base);
        for (int j = 0; j < cnt; ++j)
        {
            const double w = __shfl_sync(0xffffffffu, v, j);
            if (lane == 0) sumPsi = __dadd_rn(sumPsi, w);
        }
    }
    const double xRef = __ddiv_rn(__shfl_sync(0xffffffffu, sumPsi, 0), static_cast<double>(A.n));
    double s = 0.0;
    for (int base = 0; base < A.n; base += 32)
    {
        const int c = base + lane;
        double term = 0.0;
        if (c < A.n)
        {
            const int i = posOf[c];
            double sumA = A.diag[i];
            for (int e = A.rowStart[i]; e < A.rowStart[i + 1]; ++e) sumA = __dadd_rn(sumA, A.val[e]);
            sumA = pairRowSum(A, i, sumA);
            const double t = __dmul_rn(sumA, xRef);
            term = __dadd_rn(fabs(__dsub_rn(Apsi[i], t)), fabs(__dsub_rn(source[i], t)));
        }
        const int cnt = min(32, A.n - base);
        for (int j = 0; j < cnt; ++j)
        {
            const double v = __shfl_sync(0xffffffffu, term, j);
            if (lane == 0) s = __dadd_rn(s, v);
        }
    }
    if (lane == 0) *out = __dadd_rn(s, 1e-20);
}

// One row of a multicolour Gauss-Seidel sweep in the colour-major sliced-ELL layout (hierarchy.cuh
// Colouring): psi[p] = (b[p] - sum val*psi[col]) / diag, the entries in layout order. Every load that
// does not depend on the row's position (its slice bounds, its diagonal) and four entries' columns and
// coefficients at a time are issued before they are used, so a thread waits about four memory
// latencies per row rather than one per entry; on the small levels, where a few threads sweep a colour
// each, that latency chain is the sweep's time. The arithmetic order is the plain loop's.
// Row r < nRows: the layout pads each colour to whole slices of 32, so r's slice and its successor
// bound exist whatever pos[r] holds.
__device__ __forceinline__ void mcRowUpdate(int r, const int* __restrict__ pos, const int* __restrict__ sliceBase,
                                            const int* __restrict__ col, const float* __restrict__ val,
                                            const float* __restrict__ diag, const float* __restrict__ b,
                                            float* __restrict__ psi)
{
    const int sl = r >> 5;
    const int p = pos[r];
    const int base = sliceBase[sl];
    const int end = sliceBase[sl + 1];
    const float d = diag[r];
    if (p < 0) return;
    const int w = (end - base) >> 5;
    float acc = b[p];
    int e = base + (r & 31);
    int q = 0;
    for (; q + 4 <= w; q += 4, e += 128)
    {
        const int c0 = col[e], c1 = col[e + 32], c2 = col[e + 64], c3 = col[e + 96];
        const float v0 = val[e], v1 = val[e + 32], v2 = val[e + 64], v3 = val[e + 96];
        const float x0 = psi[c0], x1 = psi[c1], x2 = psi[c2], x3 = psi[c3];
        acc = fmaf(-v0, x0, acc);
        acc = fmaf(-v1, x1, acc);
        acc = fmaf(-v2, x2, acc);
        acc = fmaf(-v3, x3, acc);
    }
    for (; q < w; ++q, e += 32) acc = fmaf(-val[e], psi[col[e]], acc);
    psi[p] = acc / d;
}

// One colour of a multicolour Gauss-Seidel sweep (FP32 V-cycle): rows [rowBegin, rowEnd) of the
// level's colour-major sliced-ELL layout (hierarchy.cuh Colouring), one thread per row. No two rows
// of a colour share a face, so every value a row reads is final for this colour.
__global__ void mcSweep(int rowBegin, int rowEnd, const int* __restrict__ pos, const int* __restrict__ sliceBase,
                        const int* __restrict__ col, const float* __restrict__ val, const float* __restrict__ diag,
                        const float* __restrict__ b, float* __restrict__ psi);

// Every sweep of a small level's multicolour smoothing in ONE block: the colours one after another,
// a block barrier between them (levels of at most kMcSmallRows rows).
constexpr int kMcSmallRows = 65536;  // the largest level the tuner tries to sweep in one block
__global__ void mcSmoothSmall(int nColours, const int* __restrict__ colourStart, int nSweeps, int symmetric,
                              const int* __restrict__ pos, const int* __restrict__ sliceBase,
                              const int* __restrict__ col, const float* __restrict__ val,
                              const float* __restrict__ diag, const float* __restrict__ b, float* __restrict__ psi);

// The same in one thread-block cluster (mid-size levels): the cluster's CTAs share each colour's rows
// and meet at the cluster barrier (release/acquire at cluster scope) between colours. The CTAs of a
// cluster are resident together by construction, so the barrier always completes. Launched with a
// cluster dimension equal to the grid (kMcClusterMaxRows rows at most).
constexpr int kMcClusterMaxRows = 262144;
__global__ void mcSmoothCluster(int nColours, const int* __restrict__ colourStart, int nSweeps, int symmetric,
                                const int* __restrict__ pos, const int* __restrict__ sliceBase,
                                const int* __restrict__ col, const float* __restrict__ val,
                                const float* __restrict__ diag, const float* __restrict__ b, float* __restrict__ psi);

// The FP32 coefficients of the multicolour layout: per entry upper[face] (0 for padding), per row
// the diagonal at its position.
__global__ void mcValues(long long nEnt, int nRows, const int* __restrict__ face, const int* __restrict__ pos,
                         const double* __restrict__ upper, const float* __restrict__ posDiag, float* __restrict__ val,
                         float* __restrict__ diag);

}  // namespace k
}  // namespace b2g
